// gb_batch.cuh -- batched scoring and branch optimisation of many candidate
// trees (4-state data) in one persistent kernel.
//
// GARLI scores the candidates of a GA generation one at a time: each mutated
// individual recomputes its dirty CLAs (Tree::Score, tree.cpp:4003) and then
// optimises the branches around the move (OptimizeBranchesWithinRadius,
// optimization.cpp:882-884: nd->left, nd, nd->right, each by
// NewtonRaphsonOptimizeBranchLength, :1359-1971).  Here a whole batch of
// candidates runs as one cooperative launch over a device command queue:
//   kBLevel  : one dependency level of CLA updates of every candidate
//              (uneven per-candidate counts are simply concatenated), work
//              items = (op, run of pattern tiles);
//   kBNewton : Newton-Raphson on one branch of every candidate in lockstep.
//              Per iteration: (A) every active candidate's edge sweep, work
//              items = (candidate, run of 256-pattern chunks), chunk sums to
//              global memory; grid barrier; (B) one warp per active
//              candidate reduces its chunk sums in a fixed order, takes
//              gb::nr_step in FP64, recomputes P/dP/d2P at the new length and
//              re-enters the active list unless it finished; grid barrier.
//   kBScore  : lnL of every candidate at its current lengths (same sweep, no
//              Newton step).
// The chunk partition is fixed (256 patterns, one per thread), so the sums --
// and every Newton decision -- do not depend on how many chunks or tiles a
// work item covers; those run lengths are the autotuned "sites per CTA".
#pragma once
#include "gb_persist.cuh"

namespace gb {

enum BatchCmdType : int { kBLevel = 1, kBNewton = 2, kBScore = 3 };

struct BCmd {
    int type;
    int a, b;  // level: ops [a, a+b) | newton / score: entries [a, a+b)
};

// one candidate's branch: partial CLA buffer, child buffer (tip if tip != 0), matrix
struct BEntry {
    int pbuf, cbuf, tip, mat;
};

// per-entry results
struct BSlot {
    NrState st;
    double first_lnL, lnL, d1, d2, score;
    int evals;
};

struct BatchArgs {
    const BCmd *cmds;
    int ncmd;
    const DevOp *ops;
    const BEntry *entries;
    BSlot *slots;
    NrParams prm;
    double *lengths;
    const double *eig;
    const double *rates;
    double *chunk_sums;  // (entries of the largest command) x nchunks x 3
    int *active;         // 2 x (entries of the largest command)
    int *nactive;        // 2 counters
    int max_entries;
    GridSync *gs;
    int tiles_per_item;   // CLA work item: this many 64-pattern tiles
    int chunks_per_item;  // edge work item: this many 256-pattern chunks
    unsigned long long *trace;  // optional phase timestamps of block 0: (code << 56) | ns
    int trace_cap;
};

enum BatchTrace : int { kBtLevel = 1, kBtNewton, kBtSweepDone, kBtStepDone, kBtCmdDone };

constexpr int kChunk = kThreads;  // patterns per edge chunk (one per thread)

// P, dP, d2P of all R categories at length t, written by one warp to global
// memory (the operation order of pmat4_smem / Model::CalcDerivatives)
template <int R>
__device__ __forceinline__ void pmat4_warp(const double *eig, const double *rates, double pinv, int has_pinv,
                                           double t, double *out) {
    const int lane = threadIdx.x & 31;
    const double *lam = eig, *U = eig + 4, *Ui = U + 16;
    for (int idx = lane; idx < R * 16; idx += 32) {
        const int r = idx / 16, ij = idx % 16, i = ij / 4, j = ij % 4;
        double sp = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            double sev = mul(__ldcg(lam + k), __ldcg(rates + r));
            if (has_pinv) sev = sev / sub(1.0, pinv);
            const double e = exp(mul(sev, t));
            const double d1e = mul(sev, e), d2e = mul(sev, d1e);
            const double x = mul(__ldcg(U + i * 4 + k), __ldcg(Ui + k * 4 + j));
            sp = add(sp, mul(x, e));
            s1 = add(s1, mul(x, d1e));
            s2 = add(s2, mul(x, d2e));
        }
        out[idx] = sp > 0.0 ? sp : 0.0;
        out[R * 16 + idx] = s1;
        out[2 * R * 16 + idx] = s2;
    }
}

// Sweep of one edge over chunks [c0, c1) of one candidate: chunk sums to `sums`.
template <int R, bool GARLI_SCALE>
__device__ __forceinline__ void batch_edge_chunks(const View &v, const EdgeSmem<R, true> &sm, const BEntry &en,
                                                  int c0, int c1, double *sums) {
    for (int c = c0; c < c1; c++) {
        double aL = 0.0, a1 = 0.0, a2 = 0.0;
        const int p = c * kChunk + threadIdx.x;
        if (p < v.npat) {
            edge4_site_cg<double, R, GARLI_SCALE>(v, sm, en.pbuf, en.cbuf, en.tip, p, aL, a1, a2);  // plain form: FP64
        }
        block_sum3(aL, a1, a2, sums + 3 * c);
        __syncthreads();
    }
}

// Fixed-order sum of n chunk sums by one warp (lane-strided, then a shuffle tree).
__device__ __forceinline__ void warp_sum_chunks(const double *sums, int n, double &L, double &d1, double &d2) {
    const int lane = threadIdx.x & 31;
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = lane; i < n; i += 32) {
        a += __ldcg(sums + 3 * i);
        b += __ldcg(sums + 3 * i + 1);
        c += __ldcg(sums + 3 * i + 2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    L = a;
    d1 = b;
    d2 = c;
}

template <int R>
__device__ __forceinline__ void load_entry_smem(const View &v, int mat, EdgeSmem<R, true> &sm) {
    const double *mp = v.mats + (long long)mat * v.mat_stride;
    __syncthreads();
    for (int i = threadIdx.x; i < R * 16; i += blockDim.x) {
        sm.M[0][i] = __ldcg(mp + i);
        sm.M[1][i] = __ldcg(mp + R * 16 + i);
        sm.M[2][i] = __ldcg(mp + 2 * R * 16 + i);
    }
    if (threadIdx.x < 4) sm.F[threadIdx.x] = v.freqs[threadIdx.x];
    if (threadIdx.x < R) sm.RP[threadIdx.x] = v.rate_probs[threadIdx.x];
    __syncthreads();
}

template <int R, bool GARLI_SCALE>
__global__ void __launch_bounds__(kThreads, 2) k_batch4(View v, BatchArgs A) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    __shared__ EdgeSmem<R, true> sm;
    const int lane_r = threadIdx.x % G;
    const int rr = lane_r < R ? lane_r : 0;
    const int ntiles = (v.npat + PPB - 1) / PPB;
    const int nchunks = (v.npat + kChunk - 1) / kChunk;
    const int warps_per_block = blockDim.x / 32;
    const int gwarp = blockIdx.x * warps_per_block + threadIdx.x / 32;
    const int nwarps = gridDim.x * warps_per_block;
    int ntr = 0;
    auto mark = [&](int code, int na) {
        if (A.trace && blockIdx.x == 0 && threadIdx.x == 0 && ntr < A.trace_cap)
            A.trace[ntr++] = ((unsigned long long)code << 56) | ((unsigned long long)(na & 0xffff) << 40) |
                             (global_ns() & ((1ULL << 40) - 1));
    };
    for (int ci = 0; ci < A.ncmd; ci++) {
        const BCmd cmd = A.cmds[ci];
        mark(cmd.type == kBLevel ? kBtLevel : kBtNewton, cmd.b);
        if (cmd.type == kBLevel) {
            const int tpi = A.tiles_per_item;
            const int items_per_op = (ntiles + tpi - 1) / tpi;
            const long long nitems = (long long)cmd.b * items_per_op;
            int cur = -1;
            double PL[16], PR[16];
            for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
                const int j = (int)(item / items_per_op);
                const int t0 = (int)(item % items_per_op) * tpi;
                const DevOp op = A.ops[cmd.a + j];
                if (j != cur) {
                    cur = j;
                    const double *m1 = v.mats + (long long)op.p1 * v.mat_stride + 16 * rr;
                    const double *m2 = v.mats + (long long)op.p2 * v.mat_stride + 16 * rr;
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        PL[i] = __ldcg(m1 + i);
                        PR[i] = __ldcg(m2 + i);
                    }
                }
                const int t1 = min(ntiles, t0 + tpi);
                for (int tile = t0; tile < t1; tile++) {
                    cla4_tile_cg<double, R, GARLI_SCALE>(v, op, PL, PR, tile);  // plain form: FP64
                }
            }
            if (!grid_barrier(A.gs, v.status)) return;
            mark(kBtCmdDone, 0);
            continue;
        }
        // Newton / score over entries [a, a+n)
        const int n = cmd.b;
        const BEntry *ents = A.entries + cmd.a;
        BSlot *slots = A.slots + cmd.a;
        const bool newton = cmd.type == kBNewton;
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
            if (newton) {
                nr_init(slots[e].st, __ldcg(A.lengths + ents[e].mat), A.prm.min_brlen, A.prm.max_brlen);
                slots[e].evals = 0;
            }
            A.active[e] = e;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            A.nactive[0] = n;
            A.nactive[1] = 0;
        }
        if (!grid_barrier(A.gs, v.status)) return;
        int cur = 0;
        for (;;) {
            const int na = *(volatile int *)(A.nactive + cur);
            if (na == 0) break;
            const int *act = A.active + cur * A.max_entries;
            // (A) sweeps of every active entry
            const int cpi = A.chunks_per_item;
            const int items_per_entry = (nchunks + cpi - 1) / cpi;
            const long long nitems = (long long)na * items_per_entry;
            int loaded = -1;
            for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
                const int k = (int)(item / items_per_entry);
                const int c0 = (int)(item % items_per_entry) * cpi;
                const int e = __ldcg(act + k);
                const BEntry en = ents[e];
                if (e != loaded) {
                    loaded = e;
                    load_entry_smem<R>(v, en.mat, sm);
                }
                batch_edge_chunks<R, GARLI_SCALE>(v, sm, en, c0, min(nchunks, c0 + cpi),
                                                  A.chunk_sums + (long long)k * nchunks * 3);
            }
            if (!grid_barrier(A.gs, v.status)) return;
            mark(kBtSweepDone, na);
            if (blockIdx.x == 0 && threadIdx.x == 0) A.nactive[cur] = 0;  // every block has read it
            // (B) one warp per active entry: reduce, Newton step, new P
            const int nxt = cur ^ 1;
            for (int k = gwarp; k < na; k += nwarps) {
                const int e = __ldcg(act + k);
                double L, d1, d2;
                warp_sum_chunks(A.chunk_sums + (long long)k * nchunks * 3, nchunks, L, d1, d2);
                int fin = 1;
                if ((threadIdx.x & 31) == 0) {
                    BSlot &s = slots[e];
                    if (newton) {
                        if (s.evals == 0) s.first_lnL = L;
                        s.lnL = L;
                        s.d1 = d1;
                        s.d2 = d2;
                        s.evals++;
                        fin = nr_step(s.st, d1, d2, L, A.prm.precision, A.prm.min_brlen, A.prm.max_brlen);
                        A.lengths[ents[e].mat] = s.st.v;
                    } else {
                        s.score = L;
                    }
                }
                fin = __shfl_sync(0xffffffffu, fin, 0);
                if (newton) {
                    const double t = __shfl_sync(0xffffffffu, (threadIdx.x & 31) == 0 ? slots[e].st.v : 0.0, 0);
                    pmat4_warp<R>(A.eig, A.rates, v.pinv, v.has_pinv, t,
                                  const_cast<double *>(v.mats) + (long long)ents[e].mat * v.mat_stride);
                    if (!fin && (threadIdx.x & 31) == 0) {
                        const int idx = atomicAdd(A.nactive + nxt, 1);
                        A.active[nxt * A.max_entries + idx] = e;
                    }
                }
            }
            if (!grid_barrier(A.gs, v.status)) return;
            mark(kBtStepDone, na);
            cur = nxt;
        }
        // every block has left the loop before the next command resets the counters
        if (!grid_barrier(A.gs, v.status)) return;
        mark(kBtCmdDone, 0);
    }
}

}  // namespace gb
