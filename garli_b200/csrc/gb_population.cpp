// gb_population.cpp -- scoring a GA generation's candidate trees on the engine.
//
// GARLI derives each candidate of a generation from a parent tree by one
// topology move (Tree::SPRMutate, tree.cpp:3148-3248; NNI is the radius-1
// case), dirties the CLA holders the move touches (SweepDirtynessOverTree,
// tree.cpp:4247) and shares every other holder with the parent copy-on-write
// (clamanager.h numAssigned / holder reuse).  It then optimises the three
// branches around the connector node nd -- nd->left, nd, nd->right, each by
// NewtonRaphsonOptimizeBranchLength (optimization.cpp:882-884, :1359-1971).
//
// Here a CLA is identified by its content: the directional conditional
// likelihood D(v <- u) of the subtree on v's side of the branch (u, v) is
// keyed by a hash of that subtree's topology, tips and branch lengths.  The
// base tree's CLAs (all three directions of every internal node) are
// computed once; a candidate needs D(A <- X), D(B <- X), D(C <- X) for the
// connector X with neighbours A = X->left, B = X->right, C = X->anc, and only
// the keys not already present become CLA updates.  Identical subtrees are
// shared across candidates too.  A candidate keeps the base tree's node
// numbers, so only the subtrees a move changed (the nodes whose children or
// child lengths differ, and their ancestors) are hashed; the wanted CLAs are
// looked up from the top and only a missing one's sides are descended into.
// That part runs in parallel over candidates; buffers and updates are then
// assigned in candidate order.  Per step the partial on X's side of the
// optimised branch (D(X <- A), D(X <- C), D(X <- B)) is recomputed from the
// branches optimised before it.
//
// Two executions of the same plan:
//   batched    : gb_batch_newton -- every candidate in one persistent kernel;
//   sequential : GARLI's per-tree path -- per candidate its CLA updates
//                (gb_update_partials), then per branch a host Newton loop of
//                gb_calculate_edge + gb::nr_step + gb_update_transition_matrices.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../../include/garli_b200.h"
#include "gb_newton.h"

namespace {

struct Key {
    uint64_t a, b;
    bool operator==(const Key &o) const { return a == o.a && b == o.b; }
};
struct KeyHash {
    size_t operator()(const Key &k) const { return (size_t)(k.a ^ (k.b * 0x9E3779B97F4A7C15ULL)); }
};

uint64_t mix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
uint64_t bits(double d) {
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return u;
}
// key of a child term: the child's key and the length of the branch to it
Key term(const Key &child, double len) {
    const uint64_t l = bits(len);
    return {mix(child.a ^ mix(l)), mix(child.b + 0x632BE59BD9B4E019ULL * (l | 1))};
}
// order-free combination of two child terms (the CLA product is symmetric)
Key combine(const Key &x, const Key &y) {
    const Key &lo = (x.a < y.a || (x.a == y.a && x.b < y.b)) ? x : y;
    const Key &hi = (&lo == &x) ? y : x;
    return {mix(lo.a * 31 + mix(hi.a)), mix(lo.b ^ mix(hi.b + 7))};
}
Key tip_key(int t) { return {mix(0xA5A5ULL + (uint64_t)t), mix(0x5A5AULL * ((uint64_t)t + 3))}; }

struct Topo {
    int ntax = 0, nnodes = 0;
    std::vector<int> left, right, mid, anc;
    std::vector<double> dlen;
    bool tip(int n) const { return n >= 1 && n <= ntax; }
    // the three neighbours of an internal node, and the length of each branch
    int nbrs(int v, int out[3], double len[3]) const {
        int k = 0;
        if (anc[v] >= 0) {
            out[k] = anc[v];
            len[k++] = dlen[v];
        }
        for (int c : {left[v], mid[v], right[v]})
            if (c >= 0) {
                out[k] = c;
                len[k++] = dlen[c];
            }
        return k;
    }
    double blen(int a, int b) const { return anc[a] == b ? dlen[a] : dlen[b]; }
};

int load_topo(Topo &t, int ntax, const int *child3, const double *dlen) {
    t.ntax = ntax;
    t.nnodes = 2 * ntax - 2;
    const int N = t.nnodes;
    t.left.assign(N, -1);
    t.right.assign(N, -1);
    t.mid.assign(N, -1);
    t.anc.assign(N, -1);
    t.dlen.assign(dlen, dlen + N);
    int edges = 0;
    for (int i = 0; i < N; i++) {
        const int l = child3[3 * i], m = child3[3 * i + 1], r = child3[3 * i + 2];
        if (l < 0 && r < 0 && m < 0) continue;
        if (l < 0 || r < 0 || l >= N || r >= N || m >= N || (m >= 0 && i != 0) || (i >= 1 && i <= ntax))
            return GB_ERROR_OUT_OF_RANGE;
        t.left[i] = l;
        t.right[i] = r;
        t.mid[i] = m;
        for (int c : {l, m, r})
            if (c >= 0) {
                if (t.anc[c] >= 0 || c == 0) return GB_ERROR_OUT_OF_RANGE;
                t.anc[c] = i;
                edges++;
            }
    }
    if (edges != N - 1 || t.mid[0] < 0) return GB_ERROR_OUT_OF_RANGE;
    for (int i = 1; i < N; i++)
        if (t.anc[i] < 0 || !(t.dlen[i] >= 0.0)) return GB_ERROR_OUT_OF_RANGE;
    return GB_SUCCESS;
}

struct Cla {
    int buf;    // engine buffer index
    int level;  // dependency level of the op that made it (0: tip or already computed)
};

// a CLA a candidate needs that the base tree does not hold, after its
// children's: its key, its children's keys (or tip buffers) and branch lengths
struct Miss {
    Key key, k1, k2;
    int tip1, tip2;  // the child's tip buffer, or -1
    double l1, l2;
};
// what a candidate needs: its connector's three sides (A, C, B) and the
// missing CLAs, children first
struct CandNeed {
    int rc = GB_SUCCESS;
    Key side_key[3];
    int side_tip[3];
    double side_len[3];
    std::vector<Miss> miss;
};

struct Pop {
    int inst = -1;
    int ntip = 0, nbuf = 0, nmat = 0;
    Topo base;
    int rescaleEvery = 16;
    double minBrlen = 1e-8, maxBrlen = 100.0;  // defs.h:106-107
    bool base_ready = false;
    std::unordered_map<Key, Cla, KeyHash> cla;  // base CLAs (persist) + this call's
    int base_bufs = 0, next_buf = 0;
    std::unordered_map<uint64_t, int> mat_of;  // length bits -> matrix slot
    int base_mats = 0, next_mat = 0;
    std::vector<double> mat_len;
    bool wide_alloc = false;       // new CLAs of the base tree go to FP64 (two-slot) buffers
    int base_mode = -1;            // the mode the base tree was prepared for: 1 batched, 0 per-tree
    std::vector<int> wide_bufs;    // buffers currently marked FP64
    long long c_ops = 0, c_updates = 0, c_evals = 0, c_base_ops = 0, c_edges = 0;
    double c_bytes = 0.0;
    double c_bytes3[3] = {0.0, 0.0, 0.0};  // of c_bytes: CLA levels, coefficient passes, sweeps
    int npat = 0, ncat = 1;
    std::vector<Key> base_down;  // key of every node's subtree in the base tree (rooted at node 0)
    std::vector<CandNeed> needs; // planning storage, one per candidate (reused)
};

std::mutex g_mu;
std::vector<Pop *> g_pops;

Pop *get(int h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h < 0 || h >= (int)g_pops.size()) return nullptr;
    return g_pops[h];
}

// matrix slot holding P(len); shared by equal lengths
int mat_slot(Pop &p, double len, int *rc) {
    auto it = p.mat_of.find(bits(len));
    if (it != p.mat_of.end()) return it->second;
    if (p.next_mat >= p.nmat) {
        *rc = GB_ERROR_OUT_OF_RANGE;
        return 0;
    }
    const int m = p.next_mat++;
    p.mat_of[bits(len)] = m;
    p.mat_len[m] = len;
    return m;
}
int fresh_mat(Pop &p, double len, int *rc) {
    if (p.next_mat >= p.nmat) {
        *rc = GB_ERROR_OUT_OF_RANGE;
        return 0;
    }
    const int m = p.next_mat++;
    p.mat_len[m] = len;
    return m;
}

struct Made {
    Key key;
    Cla cla;
};

// D(v <- u): its key and buffer; if absent, the CLA update producing it is
// appended to ops (children first) with level 1 + the children's levels.
Made need_key(Pop &p, const Topo &t, int v, int u, std::vector<gb_cla_operation> &ops, int *rc) {
    if (t.tip(v)) return {tip_key(v), {v - 1, 0}};
    int nb[3];
    double ln[3];
    const int k = t.nbrs(v, nb, ln);
    int ch[2], c = 0;
    double cl[2];
    for (int i = 0; i < k; i++)
        if (nb[i] != u) {
            ch[c] = nb[i];
            cl[c++] = ln[i];
        }
    if (c != 2) {
        *rc = GB_ERROR_OUT_OF_RANGE;
        return {{0, 0}, {0, 0}};
    }
    const Made a = need_key(p, t, ch[0], v, ops, rc);
    if (*rc) return a;
    const Made b = need_key(p, t, ch[1], v, ops, rc);
    if (*rc) return b;
    const Key key = combine(term(a.key, cl[0]), term(b.key, cl[1]));
    auto it = p.cla.find(key);
    if (it != p.cla.end()) return {key, it->second};
    const int slots = p.wide_alloc ? 2 : 1;
    if (p.next_buf + slots > p.ntip + p.nbuf) {
        *rc = GB_ERROR_OUT_OF_RANGE;
        return {key, {0, 0}};
    }
    Cla made;
    made.buf = p.next_buf;
    p.next_buf += slots;
    if (p.wide_alloc) {
        if ((*rc = gb_set_buffer_precision(p.inst, made.buf, 1))) return {key, {0, 0}};
        p.wide_bufs.push_back(made.buf);
    }
    made.level = (a.cla.level > b.cla.level ? a.cla.level : b.cla.level) + 1;
    gb_cla_operation op;
    op.destClaIndex = made.buf;
    op.childClaIndex1 = a.cla.buf;
    op.childClaIndex2 = b.cla.buf;
    op.transMatIndex1 = mat_slot(p, cl[0], rc);
    op.transMatIndex2 = mat_slot(p, cl[1], rc);
    op.opDepLevel = made.level;
    ops.push_back(op);
    p.cla[key] = made;
    return {key, made};
}

// Keys of every node's subtree (the CLA D(v <- anc v)), the same keys
// need_key computes.  base_keys: every node of the base tree, post-order from
// the root.  cand_keys: a candidate with the base's node numbering -- a node
// whose children or child branch lengths differ from the base's is changed,
// and so is every ancestor of it; only changed nodes are hashed, the others
// keep the base's key.
void hash_node(const Topo &t, int v, std::vector<Key> &down) {
    Key terms[3];
    int k = 0;
    for (int c : {t.left[v], t.mid[v], t.right[v]})
        if (c >= 0) terms[k++] = term(down[c], t.dlen[c]);
    // the root's key (three children) is never used as a CLA key
    down[v] = k == 2 ? combine(terms[0], terms[1]) : combine(combine(terms[0], terms[1]), terms[2]);
}
void keys_below(const Topo &t, int v, const std::vector<char> *changed, std::vector<Key> &down) {
    for (int c : {t.left[v], t.mid[v], t.right[v]})
        if (c >= 0 && !t.tip(c) && (!changed || (*changed)[c])) keys_below(t, c, changed, down);
    if (v != 0) hash_node(t, v, down);
}
void base_keys(const Topo &t, std::vector<Key> &down) {
    down.resize(t.nnodes);
    for (int v = 1; v <= t.ntax; v++) down[v] = tip_key(v);
    keys_below(t, 0, nullptr, down);
}
// per-thread working storage for one candidate's keys
struct CandScratch {
    Topo t;
    std::vector<Key> down, up;   // subtree keys; up[u] = D(anc u <- u)
    std::vector<char> changed, up_known;
};

void cand_keys(const Pop &p, CandScratch &s) {
    const Topo &b = p.base, &t = s.t;
    const int N = t.nnodes;
    s.down = p.base_down;
    s.changed.assign(N, 0);
    auto mark = [&](int v) {
        for (int w = v; w >= 0 && !s.changed[w]; w = t.anc[w]) s.changed[w] = 1;
    };
    for (int v = 0; v < N; v++) {
        if (t.left[v] != b.left[v] || t.right[v] != b.right[v] || t.mid[v] != b.mid[v]) mark(v);
        if (v > 0 && bits(t.dlen[v]) != bits(b.dlen[v])) mark(t.anc[v]);
    }
    if (s.changed[0]) keys_below(t, 0, &s.changed, s.down);
    s.up.resize(N);
    s.up_known.assign(N, 0);
}

// key of D(v <- u) in the candidate: v's subtree when u is v's parent, else
// (u a child of v) the rest of the tree seen from v, built up the path to the
// root (each such key once per candidate)
Key dir_key(CandScratch &s, int v, int u) {
    const Topo &t = s.t;
    if (t.tip(v) || t.anc[v] == u) return s.down[v];
    if (s.up_known[u]) return s.up[u];
    Key terms[2];
    int k = 0;
    if (t.anc[v] >= 0) terms[k++] = term(dir_key(s, t.anc[v], v), t.dlen[v]);
    for (int c : {t.left[v], t.mid[v], t.right[v]})
        if (c >= 0 && c != u && k < 2) terms[k++] = term(s.down[c], t.dlen[c]);
    s.up[u] = combine(terms[0], terms[1]);
    s.up_known[u] = 1;
    return s.up[u];
}

// D(v <- u): its key (or tip buffer); if the base lacks it, its sides first,
// then itself appended to cn.miss (base lookups only: read-only)
void collect(const Pop &p, CandScratch &s, int v, int u, CandNeed &cn, Key &key, int &tip) {
    const Topo &t = s.t;
    if (t.tip(v)) {
        key = tip_key(v);
        tip = v - 1;
        return;
    }
    tip = -1;
    key = dir_key(s, v, u);
    if (p.cla.count(key)) return;
    int nb[3];
    double ln[3];
    const int k = t.nbrs(v, nb, ln);
    int ch[2], c = 0;
    double cl[2];
    for (int i = 0; i < k; i++)
        if (nb[i] != u && c < 2) {
            ch[c] = nb[i];
            cl[c++] = ln[i];
        }
    if (c != 2 || k != 3) {
        cn.rc = GB_ERROR_OUT_OF_RANGE;
        return;
    }
    Miss m;
    m.key = key;
    m.l1 = cl[0];
    m.l2 = cl[1];
    collect(p, s, ch[0], v, cn, m.k1, m.tip1);
    collect(p, s, ch[1], v, cn, m.k2, m.tip2);
    cn.miss.push_back(m);
}

// every directional CLA of the base tree, computed once and kept.  wide: in
// FP64 buffers (precision form, batched pass) -- they are shared by every
// candidate, so their storage error would otherwise enter every candidate's lnL.
int prepare_base(Pop &p, bool wide) {
    p.cla.clear();
    p.mat_of.clear();
    p.next_buf = p.ntip;
    p.next_mat = 0;
    for (int b : p.wide_bufs) gb_set_buffer_precision(p.inst, b, 0);
    p.wide_bufs.clear();
    // a plain instance is FP64 throughout and has no FP64 buffer option
    p.wide_alloc = wide && p.nbuf >= 2 && gb_set_buffer_precision(p.inst, p.ntip, 0) == GB_SUCCESS;
    std::vector<gb_cla_operation> ops;
    int rc = GB_SUCCESS;
    const Topo &t = p.base;
    for (int v = 0; v < t.nnodes && !rc; v++) {
        if (t.tip(v)) continue;
        int nb[3];
        double ln[3];
        const int k = t.nbrs(v, nb, ln);
        for (int i = 0; i < k && !rc; i++) need_key(p, t, v, nb[i], ops, &rc);
    }
    const bool wide_base = p.wide_alloc;
    p.wide_alloc = false;
    if (rc) return rc;
    p.base_bufs = p.next_buf;
    p.base_mats = p.next_mat;
    base_keys(p.base, p.base_down);
    std::vector<gb_transmat_operation> tops;
    for (int m = 0; m < p.next_mat; m++) tops.push_back({m, p.mat_len[m], 0, 1});
    if ((rc = gb_update_transition_matrices(p.inst, tops.data(), (int)tops.size()))) return rc;
    if (wide_base) {
        // CLA updates only, by the batched kernel (the one that reads and writes FP64 buffers)
        if ((rc = gb_batch_newton(p.inst, ops.data(), (int)ops.size(), nullptr, 0, nullptr, 0, 1, p.rescaleEvery,
                                  0.01, p.minBrlen, p.maxBrlen, nullptr)))
            return rc;
    } else if ((rc = gb_update_partials(p.inst, ops.data(), (int)ops.size(), p.rescaleEvery))) {
        return rc;
    }
    p.base_mode = wide ? 1 : 0;
    // every level of the base is computed: its CLAs have level 0 from now on
    for (auto &kv : p.cla) kv.second.level = 0;
    p.c_base_ops += (long long)ops.size();
    p.base_ready = true;
    return GB_SUCCESS;
}

// forget the previous call's CLAs and matrices (the base ones stay)
void reset_call(Pop &p) {
    for (auto it = p.cla.begin(); it != p.cla.end();)
        if (it->second.buf >= p.base_bufs) it = p.cla.erase(it);
        else ++it;
    for (auto it = p.mat_of.begin(); it != p.mat_of.end();)
        if (it->second >= p.base_mats) it = p.mat_of.erase(it);
        else ++it;
    p.next_buf = p.base_bufs;
    p.next_mat = p.base_mats;
}

struct Plan {
    std::vector<gb_cla_operation> ops;        // all candidates' dirty updates
    std::vector<int> op_owner;                // candidate whose request created each op
    std::vector<gb_cla_operation> step_ops;   // 3 per candidate
    std::vector<gb_batch_step> steps;         // 3 per candidate
    std::vector<int> nr_mat;                  // 3 per candidate (X->left, X, X->right order)
};

// Steps in GARLI's order: nd->left, nd, nd->right (optimization.cpp:882-884).
// Two phases: every candidate's keys and the CLAs the base tree lacks, in
// parallel over candidates (read-only on the base); then, in candidate order,
// the buffers, matrices and updates -- a CLA another candidate already made in
// this call is shared.  The plan is the one a serial pass would build.
int build_plan(Pop &p, int nC, const int *child3s, const double *dlens, const int *connectors, Plan &P) {
    const int N = p.base.nnodes;
    P.step_ops.resize(3 * nC);
    P.steps.resize(3 * nC);
    P.nr_mat.resize(3 * nC);
    std::vector<CandNeed> &needs = p.needs;
    needs.resize(nC);
#pragma omp parallel for schedule(static) if (nC >= 16)
    for (int c = 0; c < nC; c++) {
        thread_local CandScratch s;
        CandNeed &cn = needs[c];
        cn.rc = GB_SUCCESS;
        cn.miss.clear();
        cn.rc = load_topo(s.t, p.base.ntax, child3s + (size_t)c * 3 * N, dlens + (size_t)c * N);
        if (cn.rc) continue;
        const Topo &t = s.t;
        const int X = connectors[c];
        if (X <= t.ntax || X >= N || t.anc[X] < 0) {
            cn.rc = GB_ERROR_OUT_OF_RANGE;
            continue;
        }
        cand_keys(p, s);
        const int side[3] = {t.left[X], t.anc[X], t.right[X]};  // A, C, B
        for (int k : {0, 2, 1})  // made in the order A, B, C
            if (!cn.rc) collect(p, s, side[k], X, cn, cn.side_key[k], cn.side_tip[k]);
        cn.side_len[0] = t.dlen[t.left[X]];
        cn.side_len[1] = t.dlen[X];
        cn.side_len[2] = t.dlen[t.right[X]];
    }
    auto find = [&](const Key &key, int tip, Cla &out) -> bool {
        if (tip >= 0) {
            out = {tip, 0};
            return true;
        }
        auto it = p.cla.find(key);
        if (it == p.cla.end()) return false;
        out = it->second;
        return true;
    };
    for (int c = 0; c < nC; c++) {
        const CandNeed &cn = needs[c];
        if (cn.rc) return cn.rc;
        int rc = GB_SUCCESS;
        for (const Miss &m : cn.miss) {
            if (p.cla.count(m.key)) continue;  // made by an earlier candidate of this call
            Cla a, b;
            if (!find(m.k1, m.tip1, a) || !find(m.k2, m.tip2, b)) return GB_ERROR_OUT_OF_RANGE;
            if (p.next_buf + 1 > p.ntip + p.nbuf) return GB_ERROR_OUT_OF_RANGE;
            Cla made;
            made.buf = p.next_buf++;
            made.level = (a.level > b.level ? a.level : b.level) + 1;
            gb_cla_operation op;
            op.destClaIndex = made.buf;
            op.childClaIndex1 = a.buf;
            op.childClaIndex2 = b.buf;
            op.transMatIndex1 = mat_slot(p, m.l1, &rc);
            op.transMatIndex2 = mat_slot(p, m.l2, &rc);
            op.opDepLevel = made.level;
            if (rc) return rc;
            P.ops.push_back(op);
            P.op_owner.push_back(c);
            p.cla[m.key] = made;
        }
        Cla sides[3];
        for (int k = 0; k < 3; k++)
            if (!find(cn.side_key[k], cn.side_tip[k], sides[k])) return GB_ERROR_OUT_OF_RANGE;
        // the three branches get their own matrix slots: the device rewrites them
        const int mA = fresh_mat(p, cn.side_len[0], &rc), mC = fresh_mat(p, cn.side_len[1], &rc),
                  mB = fresh_mat(p, cn.side_len[2], &rc);
        if (rc) return rc;
        if (p.next_buf >= p.ntip + p.nbuf) return GB_ERROR_OUT_OF_RANGE;
        const int w = p.next_buf++;  // one partial buffer per candidate, rewritten at every step
        // (child buffer, its matrix) of the three sides
        const int sideBuf[3] = {sides[0].buf, sides[1].buf, sides[2].buf};
        const int sideMat[3] = {mA, mC, mB};
        for (int k = 0; k < 3; k++) {
            const int o1 = (k + 1) % 3, o2 = (k + 2) % 3;  // the two other sides
            gb_cla_operation op;
            op.destClaIndex = w;
            op.childClaIndex1 = sideBuf[o1];
            op.childClaIndex2 = sideBuf[o2];
            op.transMatIndex1 = sideMat[o1];
            op.transMatIndex2 = sideMat[o2];
            op.opDepLevel = 1;
            P.step_ops[3 * c + k] = op;
            gb_batch_step s;
            s.claOp = 3 * c + k;
            s.partialIndex = w;
            s.childIndex = sideBuf[k];
            s.transMatIndex = sideMat[k];
            P.steps[3 * c + k] = s;
            P.nr_mat[3 * c + k] = sideMat[k];
        }
    }
    return GB_SUCCESS;
}

// Algorithmic device-memory bytes of one batched pass of the precision form
// (see gbp_get_counters).
double plan_bytes(const Pop &p, const Plan &P, int nC, long long sweeps, double *parts3 = nullptr) {
    // per pattern: a CLA slice is 4R FP32 values with their extension bytes
    // and a 4-byte scale exponent (FP64 values for the parent tree's wide
    // buffers), a tip one byte; a step's coefficients are 1 + 3R doubles and a
    // scale exponent; a sweep reads those and the pattern's count and
    // constant-state word
    const double cla = 20.0 * p.ncat + 4.0, wide = 32.0 * p.ncat + 4.0;
    const double coef = 8.0 * (1 + 3 * p.ncat) + 4.0, sweep = coef + 8.0;
    auto side = [&](int b) {
        if (b < p.ntip) return 1.0;
        return (p.base_mode == 1 && !p.wide_bufs.empty() && b < p.base_bufs) ? wide : cla;
    };
    double lev = 0.0, cpass = 0.0;
    for (const gb_cla_operation &o : P.ops) lev += side(o.childClaIndex1) + side(o.childClaIndex2) + cla;
    for (int i = 0; i < 3 * nC; i++) {
        const gb_cla_operation &o = P.step_ops[i];
        cpass += coef + side(o.childClaIndex1) + side(o.childClaIndex2) + side(P.steps[i].childIndex);
    }
    const double sw = sweep * (double)sweeps;
    if (parts3) {
        parts3[0] = lev * (double)p.npat;
        parts3[1] = cpass * (double)p.npat;
        parts3[2] = sw * (double)p.npat;
    }
    return (lev + cpass + sw) * (double)p.npat;
}

int upload_mats(Pop &p) {
    int rc = gb_set_branch_lengths(p.inst, p.mat_len.data(), p.next_mat);
    if (rc) return rc;
    std::vector<gb_transmat_operation> tops;
    for (int m = p.base_mats; m < p.next_mat; m++) tops.push_back({m, p.mat_len[m], 0, 1});
    return gb_update_transition_matrices(p.inst, tops.data(), (int)tops.size());
}

// GARLI's per-tree path for one candidate's steps (host Newton loop per branch)
int run_sequential(Pop &p, const Plan &P, int nC, double prec, double *out, double *lens) {
    size_t oi = 0;
    for (int c = 0; c < nC; c++) {
        std::vector<gb_cla_operation> mine;
        while (oi < P.ops.size() && P.op_owner[oi] == c) mine.push_back(P.ops[oi++]);
        int rc = gb_update_partials(p.inst, mine.data(), (int)mine.size(), p.rescaleEvery);
        if (rc) return rc;
        p.c_ops += (long long)mine.size();
        double imp = 0.0, first = 0.0, last = 0.0;
        long long ev = 0;
        for (int k = 0; k < 3; k++) {
            const gb_batch_step &s = P.steps[3 * c + k];
            if ((rc = gb_update_partials(p.inst, &P.step_ops[3 * c + k], 1, p.rescaleEvery))) return rc;
            p.c_ops++;
            gb::NrState st;
            gb::nr_init(st, p.mat_len[s.transMatIndex], p.minBrlen, p.maxBrlen);
            gb_scoring_operation so{-1, s.partialIndex, s.childIndex, s.transMatIndex, 1};
            for (;;) {
                double r[3];
                if ((rc = gb_calculate_edge(p.inst, &so, r))) return rc;
                ev++;
                if (k == 0 && ev == 1) first = r[0];
                const int fin = gb::nr_step(st, r[1], r[2], r[0], prec, p.minBrlen, p.maxBrlen);
                if (st.v != p.mat_len[s.transMatIndex]) {
                    p.mat_len[s.transMatIndex] = st.v;
                    gb_transmat_operation t{s.transMatIndex, st.v, 0, 1};
                    if ((rc = gb_update_transition_matrices(p.inst, &t, 1))) return rc;
                }
                if (fin) break;
            }
            imp += st.totalEstImprove;
            lens[3 * c + k] = st.v;
            if (k == 2) {
                double r[3];
                so.derivatives = 0;
                if ((rc = gb_calculate_edge(p.inst, &so, r))) return rc;
                last = r[0];
            }
        }
        out[4 * c] = first;
        out[4 * c + 1] = last;
        out[4 * c + 2] = imp;
        out[4 * c + 3] = (double)ev;
        p.c_evals += ev;
    }
    return GB_SUCCESS;
}

}  // namespace

extern "C" {

int gbp_create(int instance, int ntax, const int *child3, const double *dlen, int matrixCount) {
    if (ntax < 4 || !child3 || !dlen || matrixCount < 1) return GB_ERROR_OUT_OF_RANGE;
    int shape[5];
    if (gb_get_instance_shape(instance, shape) != GB_SUCCESS) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (shape[2] != 4) return GB_ERROR_NO_IMPLEMENTATION;
    std::vector<double> probe(matrixCount);
    if (gb_get_branch_lengths(instance, probe.data(), matrixCount) != GB_SUCCESS) return GB_ERROR_OUT_OF_RANGE;
    auto *p = new Pop();
    if (load_topo(p->base, ntax, child3, dlen) != GB_SUCCESS || shape[0] < ntax) {
        delete p;
        return GB_ERROR_OUT_OF_RANGE;
    }
    p->inst = instance;
    p->ntip = shape[0];
    p->nbuf = shape[1];
    p->npat = shape[4];
    p->ncat = shape[3];
    p->nmat = matrixCount;
    p->mat_len.assign(p->nmat, 0.0);
    std::lock_guard<std::mutex> lk(g_mu);
    g_pops.push_back(p);
    return (int)g_pops.size() - 1;
}

int gbp_destroy(int pop) {
    Pop *p = get(pop);
    if (!p) return GB_ERROR_UNINITIALIZED_INSTANCE;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_pops[pop] = nullptr;
    }
    delete p;
    return GB_SUCCESS;
}

// The instance's model changed: the base CLAs are recomputed on the next call.
int gbp_invalidate(int pop) {
    Pop *p = get(pop);
    if (!p) return GB_ERROR_UNINITIALIZED_INSTANCE;
    p->base_ready = false;
    return GB_SUCCESS;
}

int gbp_score_candidates(int pop, int candidateCount, const int *child3s, const double *dlens,
                         const int *connectors, double precision, int sequential, double *out,
                         double *lengthsOut) {
    Pop *p = get(pop);
    if (!p) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (candidateCount < 1 || !child3s || !dlens || !connectors || !out || !lengthsOut || !(precision > 0.0))
        return GB_ERROR_OUT_OF_RANGE;
    for (int attempt = 0;; attempt++) {
        int rc = GB_SUCCESS;
        // the batched precision form keeps the base tree in FP64 buffers, the per-tree path cannot read them
        if (p->base_ready && (p->base_mode == 1) != (sequential == 0)) p->base_ready = false;
        if (!p->base_ready) rc = prepare_base(*p, sequential == 0);
        if (rc) return rc;
        reset_call(*p);
        Plan P;
        if ((rc = build_plan(*p, candidateCount, child3s, dlens, connectors, P))) return rc;
        if ((rc = upload_mats(*p))) return rc;
        p->c_updates = 0;
        if (sequential) {
            p->c_ops = 0;
            p->c_evals = 0;
            rc = run_sequential(*p, P, candidateCount, precision, out, lengthsOut);
            p->c_updates = p->c_ops * p->npat;
            p->c_edges = p->c_evals + candidateCount;
            p->c_bytes = plan_bytes(*p, P, candidateCount, p->c_edges, p->c_bytes3);
        } else {
            rc = gb_batch_newton(p->inst, P.ops.data(), (int)P.ops.size(), P.step_ops.data(),
                                 (int)P.step_ops.size(), P.steps.data(), candidateCount, 3, p->rescaleEvery,
                                 precision, p->minBrlen, p->maxBrlen, out);
            if (rc == GB_SUCCESS) {
                std::vector<double> len(p->next_mat);
                if ((rc = gb_get_branch_lengths(p->inst, len.data(), p->next_mat))) return rc;
                for (int i = 0; i < 3 * candidateCount; i++) lengthsOut[i] = len[P.nr_mat[i]];
                p->c_ops = (long long)P.ops.size() + (long long)P.step_ops.size();
                p->c_updates = p->c_ops * p->npat;
                p->c_evals = 0;
                for (int c = 0; c < candidateCount; c++) p->c_evals += (long long)out[4 * c + 3];
                p->c_edges = p->c_evals + candidateCount;
                p->c_bytes = plan_bytes(*p, P, candidateCount, p->c_edges, p->c_bytes3);
            }
        }
        if (rc == GB_ERROR_RESCALE_RETRY) {
            // Tree::Score's retry rule (tree.cpp:4077-4090) for the whole generation
            p->rescaleEvery -= 2;
            p->base_ready = false;
            if (p->rescaleEvery < 2) return GB_ERROR_FLOATING_POINT;
            continue;
        }
        return rc;
    }
}

int gbp_get_counters(int pop, long long *out6) {
    Pop *p = get(pop);
    if (!p) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out6[0] = p->c_ops;
    out6[1] = p->c_updates;
    out6[2] = p->c_evals;
    out6[3] = p->c_base_ops;
    out6[4] = p->c_edges;
    out6[5] = (long long)p->c_bytes;
    return GB_SUCCESS;
}

int gbp_get_byte_counters(int pop, double *out3) {
    Pop *p = get(pop);
    if (!p) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!out3) return GB_ERROR_OUT_OF_RANGE;
    for (int k = 0; k < 3; k++) out3[k] = p->c_bytes3[k];
    return GB_SUCCESS;
}

}  // extern "C"
