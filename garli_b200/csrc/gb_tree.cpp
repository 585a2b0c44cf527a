// gb_tree.cpp -- GARLI's tree-level likelihood driver on top of the engine ABI.
//
// Restates, for one data subset:
//   * the CLA holders of each internal node (treenode.h claIndexDown/UL/UR,
//     clamanager.h) with their dirty flags and SweepDirtynessOverTree
//     (tree.cpp:4247-4295);
//   * CalculationManager::CalculateLikelihoodAndDerivatives
//     (calculationmanager.cpp:476-670): collect the dirty holders a request
//     needs (AccumulateOpsOnPath), give each a dependency level, issue the
//     TransMatOperations, the level-ordered ClaOperations and one
//     ScoringOperation.  The two CLAs scored are chosen as in the CPU path
//     (Tree::ConditionalLikelihoodRateHet(ROOT), tree.cpp:3686-3811) so that the
//     engine computes exactly the CLAs GARLI's CPU build computes;
//   * Tree::Score's rescale retry loop (tree.cpp:4003-4100);
//   * NewtonRaphsonOptimizeBranchLength (optimization.cpp:1359-1971) and
//     OptimizeAllBranches / RecursivelyOptimizeBranches (optimization.cpp:97, :1042).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/garli_b200.h"
#include "gb_newton.h"

namespace {

enum { DOWN = 0, UPLEFT = 1, UPRIGHT = 2 };

struct Tree {
    int inst = -1;
    int ntax = 0, nnodes = 0;
    std::vector<int> left, right, next, anc;
    std::vector<double> dlen;
    std::vector<char> dirty;      // 3 per node
    std::vector<char> pdirty;     // P(t) of each node's branch
    std::vector<int> level;       // scratch: dep level of a holder in the current request
    std::vector<char> optimized;  // alreadyOptimized
    int rescaleEvery = 16;
    double lnL = -1.0;
    double minBrlen = 1e-8, maxBrlen = 100.0;  // defs.h:106-107
    long long nOps = 0, nPatUpdates = 0, nEdge = 0, nScores = 0, nRetries = 0;
    int npat = 0;
    bool deviceNewton = true;  // OptimizeAllBranches as one device graph (gb_newton_pass)

    bool internal(int nd) const { return nd == 0 || nd > ntax; }
    int hidx(int nd, int which) const { return nd * 3 + which; }
    // CLA buffer of holder (nd, which): internal nodes 0, ntax+1.. map to 0, 1..
    int buf(int nd, int which) const {
        const int k = nd == 0 ? 0 : nd - ntax;
        return ntax + 3 * k + which;
    }
    int tipbuf(int nd) const { return nd - 1; }
};

std::mutex g_mu;
std::vector<Tree *> g_trees;

Tree *get(int h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h < 0 || h >= (int)g_trees.size()) return nullptr;
    return g_trees[h];
}

// the two children and branch matrices of holder (nd, which) -- the operand
// choice of ConditionalLikelihoodRateHet(direction, nd), tree.cpp:3620-3683
struct Deps {
    int n1, w1;  // node and holder type of child 1 (w1 < 0: tip)
    int n2, w2;
    int m1, m2;  // nodes whose branch matrices are used
};

Deps deps_of(const Tree &t, int nd, int which) {
    Deps d;
    if (which == DOWN) {
        d.n1 = t.left[nd];
        d.n2 = t.right[nd];
        d.w1 = t.internal(d.n1) ? DOWN : -1;
        d.w2 = t.internal(d.n2) ? DOWN : -1;
        d.m1 = d.n1;
        d.m2 = d.n2;
        return d;
    }
    const int a = t.anc[nd];
    if (a >= 0) {
        d.n1 = a;
        if (t.left[a] == nd) d.w1 = UPLEFT;
        else if (t.right[a] == nd) d.w1 = UPRIGHT;
        else d.w1 = DOWN;
        d.m1 = nd;
        d.n2 = (which == UPRIGHT) ? t.left[nd] : t.right[nd];
    } else {
        if (which == UPRIGHT) {
            d.n1 = t.left[nd];
            d.n2 = t.next[t.left[nd]];
        } else {
            d.n1 = t.next[t.left[nd]];
            d.n2 = t.right[nd];
        }
        d.w1 = t.internal(d.n1) ? DOWN : -1;
        d.m1 = d.n1;
    }
    d.w2 = t.internal(d.n2) ? DOWN : -1;
    d.m2 = d.n2;
    return d;
}

// CalculationManager::AccumulateOpsOnPath (calculationmanager.cpp:631-670)
int accumulate(Tree &t, int nd, int which, std::vector<gb_cla_operation> &ops, std::vector<int> &mats) {
    if (which < 0) return 0;
    const int h = t.hidx(nd, which);
    if (!t.dirty[h]) return 0;
    if (t.level[h] > 0) return t.level[h];
    const Deps d = deps_of(t, nd, which);
    const int l1 = accumulate(t, d.n1, d.w1, ops, mats);
    const int l2 = accumulate(t, d.n2, d.w2, ops, mats);
    const int lvl = (l1 > l2 ? l1 : l2) + 1;
    t.level[h] = lvl;
    gb_cla_operation op;
    op.destClaIndex = t.buf(nd, which);
    op.childClaIndex1 = d.w1 >= 0 ? t.buf(d.n1, d.w1) : t.tipbuf(d.n1);
    op.childClaIndex2 = d.w2 >= 0 ? t.buf(d.n2, d.w2) : t.tipbuf(d.n2);
    op.transMatIndex1 = d.m1;
    op.transMatIndex2 = d.m2;
    op.opDepLevel = lvl;
    ops.push_back(op);
    mats.push_back(d.m1);
    mats.push_back(d.m2);
    return lvl;
}

struct Request {
    int pn, pw;  // partial holder
    int cn, cw;  // child holder (cw < 0: tip)
    int mat;     // branch matrix
    bool derivs;
};

// Tree::ConditionalLikelihoodRateHet(ROOT, nd), tree.cpp:3711-3767
Request root_request(const Tree &t, int nd) {
    Request r;
    r.derivs = false;
    if (!t.dirty[t.hidx(nd, UPLEFT)]) {
        r.pn = nd;
        r.pw = UPLEFT;
        r.cn = t.left[nd];
        r.mat = r.cn;
    } else if (!t.dirty[t.hidx(nd, UPRIGHT)]) {
        r.pn = nd;
        r.pw = UPRIGHT;
        r.cn = t.right[nd];
        r.mat = r.cn;
    } else {
        r.pn = nd;
        r.pw = DOWN;
        const int a = t.anc[nd];
        if (a >= 0) {
            r.cn = a;
            if (t.left[a] == nd) r.cw = UPLEFT;
            else if (t.right[a] == nd) r.cw = UPRIGHT;
            else r.cw = DOWN;
            r.mat = nd;
            return r;
        }
        r.cn = t.next[t.left[nd]];
        r.mat = r.cn;
    }
    r.cw = t.internal(r.cn) ? DOWN : -1;
    return r;
}

// Tree::CalcDerivativesRateHet(nd->anc, nd), optimization.cpp:1112-1123
Request deriv_request(const Tree &t, int nd) {
    Request r;
    r.derivs = true;
    const int a = t.anc[nd];
    r.pn = a;
    if (t.left[a] == nd) r.pw = UPLEFT;
    else if (t.right[a] == nd) r.pw = UPRIGHT;
    else r.pw = DOWN;
    r.cn = nd;
    r.cw = t.internal(nd) ? DOWN : -1;
    r.mat = nd;
    return r;
}

void make_all_dirty(Tree &t) {
    std::fill(t.dirty.begin(), t.dirty.end(), 1);
    std::fill(t.pdirty.begin(), t.pdirty.end(), 1);
    t.lnL = -1.0;
}

// CalculateLikelihoodAndDerivatives + the rescale retry of Tree::Score
// (tree.cpp:4077-4090) / NewtonRaphsonOptimizeBranchLength (optimization.cpp:1456-1474)
int run_request(Tree &t, bool score, int node, double *out) {
    for (int attempt = 0;; attempt++) {
        const Request rq = score ? root_request(t, node) : deriv_request(t, node);
        std::vector<gb_cla_operation> ops;
        std::vector<int> mats;
        std::fill(t.level.begin(), t.level.end(), 0);
        accumulate(t, rq.pn, rq.pw, ops, mats);
        accumulate(t, rq.cn, rq.cw, ops, mats);
        mats.push_back(rq.mat);
        std::vector<gb_transmat_operation> tops;
        for (int m : mats) {
            if (!t.pdirty[m]) continue;
            t.pdirty[m] = 0;
            gb_transmat_operation o;
            o.destTransMatIndex = m;
            o.edgeLength = t.dlen[m];
            o.eigenIndex = 0;
            o.calcDerivs = 1;
            tops.push_back(o);
        }
        int rc = gb_update_transition_matrices(t.inst, tops.data(), (int)tops.size());
        if (rc) return rc;
        rc = gb_update_partials(t.inst, ops.data(), (int)ops.size(), t.rescaleEvery);
        if (rc) return rc;
        for (int nd = 0; nd < t.nnodes; nd++)
            for (int w = 0; w < 3; w++)
                if (t.level[t.hidx(nd, w)] > 0) t.dirty[t.hidx(nd, w)] = 0;
        t.nOps += (long long)ops.size();
        t.nPatUpdates += (long long)ops.size() * t.npat;
        gb_scoring_operation so;
        so.destClaIndex = -1;
        so.childClaIndex1 = t.buf(rq.pn, rq.pw);
        so.childClaIndex2 = rq.cw >= 0 ? t.buf(rq.cn, rq.cw) : t.tipbuf(rq.cn);
        so.transMatIndex = rq.mat;
        so.derivatives = rq.derivs ? 1 : 0;
        rc = gb_calculate_edge(t.inst, &so, out);
        t.nEdge++;
        if (rc == GB_ERROR_RESCALE_RETRY) {
            t.nRetries++;
            make_all_dirty(t);
            t.rescaleEvery -= 2;
            if (t.rescaleEvery < 2) return GB_ERROR_FLOATING_POINT;
            continue;
        }
        if (rc) return rc;
        t.lnL = out[0];
        if (score) t.nScores++;
        return GB_SUCCESS;
    }
}

// SweepDirtynessOverTree, tree.cpp:4247-4295
void sweep(Tree &t, int nd, int from) {
    t.lnL = -1.0;
    auto D = [&](int n, int w) { t.dirty[t.hidx(n, w)] = 1; };
    if (from < 0) {
        if (t.internal(nd)) {
            D(nd, UPLEFT);
            D(nd, UPRIGHT);
            if (t.internal(t.left[nd])) sweep(t, t.left[nd], nd);
            if (t.internal(t.right[nd])) sweep(t, t.right[nd], nd);
        }
        if (t.anc[nd] >= 0) sweep(t, t.anc[nd], nd);
        return;
    }
    if (from == t.anc[nd] || (nd == 0 && from == t.next[t.left[nd]])) {
        D(nd, UPLEFT);
        D(nd, UPRIGHT);
        if (t.internal(t.left[nd])) sweep(t, t.left[nd], nd);
        if (t.internal(t.right[nd])) sweep(t, t.right[nd], nd);
    } else if (from == t.left[nd]) {
        D(nd, UPRIGHT);
        D(nd, DOWN);
        if (t.internal(t.right[nd])) sweep(t, t.right[nd], nd);
        if (t.anc[nd] >= 0) sweep(t, t.anc[nd], nd);
        else if (t.internal(t.next[t.left[nd]])) sweep(t, t.next[t.left[nd]], nd);
    } else if (from == t.right[nd]) {
        D(nd, UPLEFT);
        D(nd, DOWN);
        if (t.internal(t.left[nd])) sweep(t, t.left[nd], nd);
        if (t.anc[nd] >= 0) sweep(t, t.anc[nd], nd);
        else if (t.internal(t.next[t.left[nd]])) sweep(t, t.next[t.left[nd]], nd);
    }
}

void set_blen(Tree &t, int nd, double v) {
    t.dlen[nd] = v;
    t.pdirty[nd] = 1;
    sweep(t, nd, -1);
}

bool fp_equals(double a, double b, double eps) { return std::fabs(a - b) < eps; }

int score(Tree &t, int root, double *lnl) {
    double out[3];
    int rc = run_request(t, true, root, out);
    if (lnl) *lnl = out[0];
    return rc;
}

// NewtonRaphsonOptimizeBranchLength, optimization.cpp:1359-1971: derivative
// evaluations on the engine, one gb::nr_step per iteration (gb_newton.h).
int nr_optimize(Tree &t, double precision1, int nd, double *result) {
    gb::NrState st;
    gb::nr_init(st, t.dlen[nd], t.minBrlen, t.maxBrlen);
    double out[3];
    for (;;) {
        int rc = run_request(t, false, nd, out);
        if (rc) return rc;
        const int fin = gb::nr_step(st, out[1], out[2], out[0], precision1, t.minBrlen, t.maxBrlen);
        if (st.v != t.dlen[nd]) set_blen(t, nd, st.v);
        if (fin) break;
    }
    *result = st.totalEstImprove;
    return GB_SUCCESS;
}

// RecursivelyOptimizeBranches, optimization.cpp:1042-1062
int rec_opt(Tree &t, int nd, double prec, int radius, bool dontGoNext, bool ignoreDelta, double *acc) {
    double delta = 0.0;
    if (!t.optimized[nd]) {
        t.optimized[nd] = 1;
        int rc = nr_optimize(t, prec, nd, &delta);
        if (rc) return rc;
    }
    *acc += delta;
    if (t.left[nd] >= 0 && radius > 1 && (!(delta < prec) || ignoreDelta)) {
        int rc = rec_opt(t, t.left[nd], prec, radius - 1, false, ignoreDelta, acc);
        if (rc) return rc;
    }
    if (t.next[nd] >= 0 && !dontGoNext && !t.optimized[t.next[nd]]) {
        int rc = rec_opt(t, t.next[nd], prec, radius, false, ignoreDelta, acc);
        if (rc) return rc;
    }
    return GB_SUCCESS;
}

// Traversal order of OptimizeAllBranches -> RecursivelyOptimizeBranches with
// ignoreDelta = true and an unbounded radius (optimization.cpp:97-105, :1042-1062)
void pass_order(const Tree &t, int nd, bool dontGoNext, std::vector<int> &order, std::vector<char> &seen) {
    if (!seen[nd]) {
        seen[nd] = 1;
        order.push_back(nd);
    }
    if (t.left[nd] >= 0) pass_order(t, t.left[nd], false, order, seen);
    if (t.next[nd] >= 0 && !dontGoNext && !seen[t.next[nd]]) pass_order(t, t.next[nd], false, order, seen);
}

// OptimizeAllBranches as one device graph.  The plan assumes every branch
// moves: its sweep (SweepDirtynessOverTree) is applied after each branch, so
// a CLA that GARLI would have reused is recomputed from identical inputs
// instead, which gives identical values.
int optimize_all_device(Tree &t, double prec, double *out) {
    for (;;) {
        const std::vector<double> dlen0 = t.dlen;
        const std::vector<char> dirty0 = t.dirty, pdirty0 = t.pdirty;
        int rc = gb_set_branch_lengths(t.inst, t.dlen.data(), t.nnodes);
        if (rc) return rc;
        std::vector<gb_transmat_operation> tops;
        for (int m = 1; m < t.nnodes; m++) {
            if (!t.pdirty[m]) continue;
            gb_transmat_operation o;
            o.destTransMatIndex = m;
            o.edgeLength = t.dlen[m];
            o.eigenIndex = 0;
            o.calcDerivs = 1;
            tops.push_back(o);
            t.pdirty[m] = 0;
        }
        rc = gb_update_transition_matrices(t.inst, tops.data(), (int)tops.size());
        if (rc) return rc;
        std::vector<int> order;
        std::vector<char> seen(t.nnodes, 0);
        const int l = t.left[0], m = t.next[l], r = t.right[0];
        for (int c : {l, m, r}) pass_order(t, c, true, order, seen);
        std::vector<gb_nr_branch> br;
        std::vector<gb_cla_operation> ops;
        std::vector<int> mats;
        for (int nd : order) {
            const Request rq = deriv_request(t, nd);
            std::fill(t.level.begin(), t.level.end(), 0);
            const int first = (int)ops.size();
            accumulate(t, rq.pn, rq.pw, ops, mats);
            accumulate(t, rq.cn, rq.cw, ops, mats);
            for (int q = 0; q < t.nnodes; q++)
                for (int w = 0; w < 3; w++)
                    if (t.level[t.hidx(q, w)] > 0) t.dirty[t.hidx(q, w)] = 0;
            gb_nr_branch b;
            b.partialIndex = t.buf(rq.pn, rq.pw);
            b.childIndex = rq.cw >= 0 ? t.buf(rq.cn, rq.cw) : t.tipbuf(rq.cn);
            b.transMatIndex = nd;
            b.firstOp = first;
            b.opCount = (int)ops.size() - first;
            br.push_back(b);
            sweep(t, nd, -1);
        }
        double res[3];
        rc = gb_newton_pass(t.inst, br.data(), (int)br.size(), ops.data(), (int)ops.size(), t.rescaleEvery, prec,
                            t.minBrlen, t.maxBrlen, res);
        if (rc == GB_ERROR_RESCALE_RETRY) {
            // Tree::Score / NR retry rule (tree.cpp:4077-4090): lower rescaleEvery and redo
            t.nRetries++;
            t.dlen = dlen0;
            t.dirty = dirty0;
            t.pdirty = pdirty0;
            make_all_dirty(t);
            t.rescaleEvery -= 2;
            if (t.rescaleEvery < 2) return GB_ERROR_FLOATING_POINT;
            continue;
        }
        if (rc) return rc;
        rc = gb_get_branch_lengths(t.inst, t.dlen.data(), t.nnodes);
        if (rc) return rc;
        t.nOps += (long long)ops.size();
        t.nPatUpdates += (long long)ops.size() * t.npat;
        t.nEdge += (long long)res[2];
        t.lnL = -1.0;
        out[0] = res[0];
        out[1] = res[1];
        return GB_SUCCESS;
    }
}

// Tree::Score after MakeAllNodesDirty under count models at once (one
// SetAndEvaluateParameter per model, optimization.cpp:244-268): model k reads
// eigen / model slot slots[k], its P(t) in matrices (k+1)*nnodes + node and
// its Down CLAs in buffers past the tree's own 3 per internal node.  The
// operations of all models go to the engine as one levelled list, the root
// edges as one gb_calculate_edges call; the tree's own CLAs and P(t) are not
// touched.  The CLAs scored are those of the root request at node 0 with
// every holder dirty (root_request): Down(0) against the middle child's Down.
int score_models(Tree &t, int count, const int *slots, double *lnl) {
    int cap[3];
    int rc = gb_get_instance_capacity(t.inst, cap);
    if (rc) return rc;
    const int nint = t.ntax - 2;
    if (cap[0] < 3 * nint + count * nint || cap[1] < (count + 1) * t.nnodes) return GB_ERROR_OUT_OF_RANGE;
    for (int k = 0; k < count; k++)
        if (slots[k] < 0 || slots[k] >= cap[2]) return GB_ERROR_OUT_OF_RANGE;
    auto kbuf = [&](int k, int nd) { return t.ntax + 3 * nint + k * nint + (nd == 0 ? 0 : nd - t.ntax); };
    auto kmat = [&](int k, int nd) { return (k + 1) * t.nnodes + nd; };
    // dependency level of each internal node's Down holder (tips: 0), as accumulate() numbers them
    std::vector<int> lvl(t.nnodes, 0), post;
    std::vector<int> stack{0};
    while (!stack.empty()) {
        const int nd = stack.back();
        stack.pop_back();
        post.push_back(nd);
        for (int c = t.left[nd]; c >= 0; c = t.next[c])
            if (t.internal(c)) stack.push_back(c);
    }
    for (int i = (int)post.size() - 1; i >= 0; i--) {
        const int nd = post[i];
        const Deps d = deps_of(t, nd, DOWN);
        lvl[nd] = std::max(d.w1 >= 0 ? lvl[d.n1] : 0, d.w2 >= 0 ? lvl[d.n2] : 0) + 1;
    }
    const int mid = t.next[t.left[0]];
    for (;;) {
        std::vector<gb_transmat_operation> tops;
        std::vector<gb_cla_operation> ops;
        std::vector<gb_scoring_operation> sops(count);
        for (int k = 0; k < count; k++) {
            for (int nd = 1; nd < t.nnodes; nd++) {
                gb_transmat_operation o;
                o.destTransMatIndex = kmat(k, nd);
                o.edgeLength = t.dlen[nd];
                o.eigenIndex = slots[k];
                o.calcDerivs = 0;
                tops.push_back(o);
            }
            for (int nd : post) {
                const Deps d = deps_of(t, nd, DOWN);
                gb_cla_operation op;
                op.destClaIndex = kbuf(k, nd);
                op.childClaIndex1 = d.w1 >= 0 ? kbuf(k, d.n1) : t.tipbuf(d.n1);
                op.childClaIndex2 = d.w2 >= 0 ? kbuf(k, d.n2) : t.tipbuf(d.n2);
                op.transMatIndex1 = kmat(k, d.m1);
                op.transMatIndex2 = kmat(k, d.m2);
                op.opDepLevel = lvl[nd];
                ops.push_back(op);
            }
            gb_scoring_operation &so = sops[k];
            so.destClaIndex = -1;
            so.childClaIndex1 = kbuf(k, 0);
            so.childClaIndex2 = t.internal(mid) ? kbuf(k, mid) : t.tipbuf(mid);
            so.transMatIndex = kmat(k, mid);
            so.derivatives = 0;
        }
        if ((rc = gb_update_transition_matrices(t.inst, tops.data(), (int)tops.size()))) return rc;
        if ((rc = gb_update_partials(t.inst, ops.data(), (int)ops.size(), t.rescaleEvery))) return rc;
        std::vector<double> out(3 * (size_t)count);
        rc = gb_calculate_edges(t.inst, sops.data(), slots, count, out.data());
        t.nOps += (long long)ops.size();
        t.nPatUpdates += (long long)ops.size() * t.npat;
        t.nEdge += count;
        if (rc == GB_ERROR_RESCALE_RETRY) {
            // Tree::Score's retry (tree.cpp:4077-4090)
            t.nRetries++;
            make_all_dirty(t);
            t.rescaleEvery -= 2;
            if (t.rescaleEvery < 2) return GB_ERROR_FLOATING_POINT;
            continue;
        }
        if (rc) return rc;
        for (int k = 0; k < count; k++) lnl[k] = out[3 * k];
        t.nScores += count;
        return GB_SUCCESS;
    }
}

}  // namespace

extern "C" {

int gbt_score_models(int tree, int count, const int *eigenIndices, double *lnl) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (count < 1 || !eigenIndices || !lnl) return GB_ERROR_OUT_OF_RANGE;
    return score_models(*t, count, eigenIndices, lnl);
}

int gbt_get_instance(int tree) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    return t->inst;
}

int gbt_create(int instance, int ntax, const int *child3, const double *dlen) {
    if (ntax < 3 || !child3 || !dlen) return GB_ERROR_OUT_OF_RANGE;
    auto *t = new Tree();
    t->inst = instance;
    t->ntax = ntax;
    t->nnodes = 2 * ntax - 2;
    const int N = t->nnodes;
    t->left.assign(N, -1);
    t->right.assign(N, -1);
    t->next.assign(N, -1);
    t->anc.assign(N, -1);
    t->dlen.assign(dlen, dlen + N);
    for (int i = 0; i < N; i++) {
        const int l = child3[3 * i], m = child3[3 * i + 1], r = child3[3 * i + 2];
        if (l < 0) continue;
        if (l >= N || r < 0 || r >= N || m >= N) {
            delete t;
            return GB_ERROR_OUT_OF_RANGE;
        }
        t->left[i] = l;
        t->right[i] = r;
        t->anc[l] = i;
        t->anc[r] = i;
        if (m >= 0) {
            t->anc[m] = i;
            t->next[l] = m;
            t->next[m] = r;
        } else {
            t->next[l] = r;
        }
    }
    t->dirty.assign(3 * N, 1);
    t->pdirty.assign(N, 1);
    t->level.assign(3 * N, 0);
    t->optimized.assign(N, 0);
    int shape[5];
    if (gb_get_instance_shape(instance, shape) != GB_SUCCESS) {
        delete t;
        return GB_ERROR_UNINITIALIZED_INSTANCE;
    }
    // the tree needs tip buffers 0..ntax-1 and 3 CLA buffers per internal node
    if (shape[0] < ntax || shape[1] < 3 * (ntax - 2)) {
        delete t;
        return GB_ERROR_OUT_OF_RANGE;
    }
    t->npat = shape[4];
    std::lock_guard<std::mutex> lk(g_mu);
    g_trees.push_back(t);
    return (int)g_trees.size() - 1;
}

int gbt_destroy(int tree) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_trees[tree] = nullptr;
    }
    delete t;
    return GB_SUCCESS;
}

int gbt_set_model(int tree, const double *eigenValues, const double *U, const double *Uinv, double blenMult,
                  const double *pi, const double *rates, const double *weights, double pinv, int hasPinv) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    int shape[5];
    int rc = gb_get_instance_shape(t->inst, shape);
    if (rc) return rc;
    const int S = shape[2];
    // eigenvalues go to the engine pre-scaled by blen_multiplier (model.cpp:845-846)
    std::vector<double> scaled(eigenValues, eigenValues + S);
    for (double &x : scaled) x *= blenMult;
    if ((rc = gb_set_eigen_decomposition(t->inst, 0, U, Uinv, scaled.data()))) return rc;
    if ((rc = gb_set_state_frequencies(t->inst, pi))) return rc;
    if ((rc = gb_set_category_rates(t->inst, rates))) return rc;
    if ((rc = gb_set_category_weights(t->inst, weights))) return rc;
    if ((rc = gb_set_invariant_sites(t->inst, pinv, hasPinv))) return rc;
    make_all_dirty(*t);
    return GB_SUCCESS;
}

int gbt_score(int tree, int rootNode, double *out) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (rootNode < 0 || rootNode >= t->nnodes || !t->internal(rootNode)) return GB_ERROR_OUT_OF_RANGE;
    return score(*t, rootNode, out);
}

int gbt_derivatives(int tree, int node, double *out) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (node <= 0 || node >= t->nnodes) return GB_ERROR_OUT_OF_RANGE;
    return run_request(*t, false, node, out);
}

int gbt_set_branch_length(int tree, int node, double length) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (node <= 0 || node >= t->nnodes || !(length >= 0.0)) return GB_ERROR_OUT_OF_RANGE;
    set_blen(*t, node, length);
    return GB_SUCCESS;
}

int gbt_get_branch_lengths(int tree, double *dlen) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    std::memcpy(dlen, t->dlen.data(), sizeof(double) * t->nnodes);
    return GB_SUCCESS;
}

int gbt_make_all_dirty(int tree) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    make_all_dirty(*t);
    return GB_SUCCESS;
}

int gbt_optimize_branch(int tree, double precision, int node, double *out) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (node <= 0 || node >= t->nnodes) return GB_ERROR_OUT_OF_RANGE;
    return nr_optimize(*t, precision, node, out);
}

int gbt_optimize_all_branches(int tree, double precision, double *out) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (t->deviceNewton) return optimize_all_device(*t, precision, out);
    std::fill(t->optimized.begin(), t->optimized.end(), 0);
    double improve = 0.0;
    const int l = t->left[0], m = t->next[l], r = t->right[0];
    for (int c : {l, m, r}) {
        int rc = rec_opt(*t, c, precision, t->nnodes, true, true, &improve);
        if (rc) return rc;
    }
    out[0] = improve;
    out[1] = t->lnL;
    return GB_SUCCESS;
}

int gbt_set_device_newton(int tree, int on) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    t->deviceNewton = on != 0;
    return GB_SUCCESS;
}

int gbt_get_rescale_every(int tree) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    return t->rescaleEvery;
}

int gbt_set_rescale_every(int tree, int every) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    t->rescaleEvery = every;
    return GB_SUCCESS;
}

int gbt_get_counters(int tree, long long *out) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out[0] = t->nOps;
    out[1] = t->nPatUpdates;
    out[2] = t->nEdge;
    out[3] = t->nScores;
    out[4] = t->nRetries;
    return GB_SUCCESS;
}

int gbt_cla_buffer(int tree, int node, int which) {
    Tree *t = get(tree);
    if (!t) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (node < 0 || node >= t->nnodes || which < 0 || which > 2 || !t->internal(node)) return GB_ERROR_OUT_OF_RANGE;
    if (t->dirty[t->hidx(node, which)]) return -1;
    return t->buf(node, which);
}

}  // extern "C"
