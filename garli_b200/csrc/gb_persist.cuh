// gb_persist.cuh -- the persistent pass kernel for 4-state data.
//
// One cooperative launch executes a device-side command queue:
//   kCmdLevel  : a dependency level of CLA updates (Tree::UpdateCLAs), all
//                blocks sharing the (op, pattern tile) work items;
//   kCmdNewton : NewtonRaphsonOptimizeBranchLength on one branch
//                (optimization.cpp:1359-1971): per iteration every block sums
//                lnL/d1/d2 over its share of the patterns, one grid barrier,
//                then every block reduces all partial sums in the same fixed
//                order, takes the same gb::nr_step and recomputes P/dP/d2P at
//                the new length in its own shared memory -- identical
//                decisions everywhere, one barrier per iteration.
// Commands are separated by grid barriers.  Data written inside the launch by
// other blocks is read through L2 (ld.global.cg), never the incoherent L1 /
// read-only path.  Every barrier wait is bounded (poll count and wall time): a
// block that gives up sets an error bit and the whole launch winds down.
#pragma once
#include "gb_dna.cuh"
#include "gb_graph.cuh"
#include "gb_pmat.cuh"

namespace gb {

enum CmdType : int { kCmdLevel = 1, kCmdNewton = 2 };
enum : int { kStatusBarrierTimeout = 4 };
constexpr long long kSpinLimit = 1LL << 26;
constexpr unsigned long long kBarrierNs = 4000000000ULL;  // 4 s

struct PCmd {
    int type;
    int a, b, c, d;  // level: first op, op count | newton: partial buf, child buf, child is tip, matrix
};

struct GridSync {
    unsigned int count;
    unsigned int gen;
};

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned int atom_add_acq_rel_gpu(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void red_release_gpu(unsigned int *p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Sense-counting grid barrier for a cooperative launch (all blocks resident):
// acquire/release atomics at GPU scope, the CTA's earlier writes ordered by a
// fence before arrival.  The wait is bounded twice (kSpinLimit polls and
// kBarrierNs of %globaltimer); a block that gives up sets an error bit, and a
// waiting block that sees the bit stops waiting, so every block returns false
// from this and later barriers and the launch winds down promptly.
__device__ __forceinline__ bool grid_barrier(GridSync *gs, int *status) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = (*(volatile int *)status & kStatusBarrierTimeout) ? 0 : 1;
        if (ok) {
            const unsigned int g = ld_acquire_gpu(&gs->gen);
            __threadfence();
            const unsigned int arrived = atom_add_acq_rel_gpu(&gs->count, 1u) + 1u;
            if (arrived == gridDim.x) {
                gs->count = 0;
                red_release_gpu(&gs->gen, 1u);
            } else {
                const unsigned long long t0 = global_ns();
                long long spins = 0;
                while (ld_acquire_gpu(&gs->gen) == g) {
                    if ((++spins & 255) == 0) {
                        if (*(volatile int *)status & kStatusBarrierTimeout) {
                            ok = 0;
                            break;
                        }
                        if (spins > kSpinLimit || global_ns() - t0 > kBarrierNs) {
                            atomicOr(status, kStatusBarrierTimeout);
                            ok = 0;
                            break;
                        }
                    }
                }
            }
            if (*(volatile int *)status & kStatusBarrierTimeout) ok = 0;
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// L2-coherent loads for data other blocks of the same launch may have written
__device__ __forceinline__ void ld4d_cg(const double *p, double v[4]) {
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
                 : "l"(p));
}
template <typename ST>
__device__ __forceinline__ void cla_load_cg(const ST *p, double v[4]);
template <>
__device__ __forceinline__ void cla_load_cg<double>(const double *p, double v[4]) { ld4d_cg(p, v); }

// P, dP, d2P of all R categories at length t into shared memory (the
// operations and their order are those of pmat_body / Model::CalcDerivatives)
template <int R>
__device__ __forceinline__ void pmat4_smem(const double *eig, const double *rates, double pinv, int has_pinv,
                                           double t, double (*M)[R * 16], double *scratch) {
    double *ex = scratch, *d1e = ex + R * 4, *d2e = d1e + R * 4;
    const double *lam = eig, *U = eig + 4, *Ui = U + 16;
    for (int idx = threadIdx.x; idx < R * 4; idx += blockDim.x) {
        const int r = idx / 4, k = idx % 4;
        double sev = mul(__ldcg(lam + k), __ldcg(rates + r));
        if (has_pinv) sev = sev / sub(1.0, pinv);
        const double e = exp(mul(sev, t));
        ex[idx] = e;
        d1e[idx] = mul(sev, e);
        d2e[idx] = mul(sev, d1e[idx]);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < R * 16; idx += blockDim.x) {
        const int r = idx / 16, ij = idx % 16, i = ij / 4, j = ij % 4;
        double sp = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const double x = mul(__ldcg(U + i * 4 + k), __ldcg(Ui + k * 4 + j));
            sp = add(sp, mul(x, ex[r * 4 + k]));
            s1 = add(s1, mul(x, d1e[r * 4 + k]));
            s2 = add(s2, mul(x, d2e[r * 4 + k]));
        }
        M[0][idx] = sp > 0.0 ? sp : 0.0;
        M[1][idx] = s1;
        M[2][idx] = s2;
    }
    __syncthreads();
}

// The edge site computation of edge4_site with L2-coherent CLA loads.
template <typename ST, int R, bool GARLI_SCALE>
__device__ __forceinline__ void edge4_site_cg(const View &v, const EdgeSmem<R, true> &sm, int pbuf, int cbuf,
                                              int child_tip, int p, double &accL, double &acc1, double &acc2) {
    const double *f = sm.F;
    double L[4] = {0, 0, 0, 0}, D1[4] = {0, 0, 0, 0}, D2[4] = {0, 0, 0, 0};
    const int m1 = __ldcg(v.scalers + (long long)pbuf * v.npat_pad + p);
    const int m2 = child_tip ? 0 : __ldcg(v.scalers + (long long)cbuf * v.npat_pad + p);
    const ST *PC = cla_ptr<ST>(v, pbuf, p, R * 4);
    if (!child_tip) {
        const ST *CC = cla_ptr<ST>(v, cbuf, p, R * 4);
#pragma unroll
        for (int r = 0; r < R; r++) {
            double part[4], c[4];
            cla_load_cg<ST>(PC + r * 4, part);
            cla_load_cg<ST>(CC + r * 4, c);
            const double rp = sm.RP[r];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                L[i] = add(L[i], mul(mul(dot4_seq(&sm.M[0][16 * r + 4 * i], c), part[i]), rp));
                D1[i] = add(D1[i], mul(mul(dot4_seq(&sm.M[1][16 * r + 4 * i], c), part[i]), rp));
                D2[i] = add(D2[i], mul(mul(dot4_seq(&sm.M[2][16 * r + 4 * i], c), part[i]), rp));
            }
        }
    } else {
        const int code = v.tips[(long long)cbuf * v.npat_pad + p] & 15;
        const int cls = tip_class(code);
        if (cls == 1) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                double part[4];
                cla_load_cg<ST>(PC + r * 4, part);
#pragma unroll
                for (int i = 0; i < 4; i++) L[i] = add(L[i], mul(part[i], sm.RP[r]));
            }
        } else {
            for (int s = 0; s < 4; s++) {
                if (!(code & (1 << s))) continue;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    double part[4];
                    cla_load_cg<ST>(PC + r * 4, part);
                    const double rp = sm.RP[r];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        L[i] = add(L[i], mul(mul(sm.M[0][16 * r + 4 * i + s], part[i]), rp));
                        D1[i] = add(D1[i], mul(mul(sm.M[1][16 * r + 4 * i + s], part[i]), rp));
                        D2[i] = add(D2[i], mul(mul(sm.M[2][16 * r + 4 * i + s], part[i]), rp));
                    }
                }
            }
        }
    }
    double siteL = add(add(add(mul(L[0], f[0]), mul(L[1], f[1])), mul(L[2], f[2])), mul(L[3], f[3]));
    const int cb = v.const_states[p];
    if (v.has_pinv && cb >= 0) {
        double btot = 0.0;
        if (cb & 1) btot = add(btot, f[0]);
        if (cb & 2) btot = add(btot, f[1]);
        if (cb & 4) btot = add(btot, f[2]);
        if (cb & 8) btot = add(btot, f[3]);
        if (GARLI_SCALE) {
            const double e = child_tip ? exp((double)m1) : exp(add((double)m2, (double)m1));
            siteL = add(siteL, mul(mul(v.pinv, btot), e));
        } else {
            siteL = add(siteL, ldexp(mul(v.pinv, btot), m1 + m2));
        }
    }
    double u;
    if (GARLI_SCALE) {
        const double lg = log(siteL);
        if (!child_tip) u = sub(sub(lg, (double)m2), (double)m1);
        else u = sub(sub(lg, (double)m1), (double)m2);
    } else {
        u = sub(log(siteL), (double)(m1 + m2) * 0.69314718055994530941723212145818);
    }
    const double cnt = (double)v.counts[p];
    accL = add(accL, mul(cnt, u));
    const double sd1 = add(add(add(mul(D1[0], f[0]), mul(D1[1], f[1])), mul(D1[2], f[2])), mul(D1[3], f[3])) / siteL;
    const double sd2 =
        sub(add(add(add(mul(D2[0], f[0]), mul(D2[1], f[1])), mul(D2[2], f[2])), mul(D2[3], f[3])) / siteL,
            mul(sd1, sd1));
    acc1 = add(acc1, mul(cnt, sd1));
    acc2 = add(acc2, mul(cnt, sd2));
}

// CLA tile of cla4_body with L2-coherent loads of the children and scalers
template <typename ST, int R, bool GARLI_SCALE>
__device__ __forceinline__ void cla4_tile_cg(const View &v, const DevOp &op, const double *PL, const double *PR,
                                             int tile) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    const int r = threadIdx.x % G;
    const int p = tile * PPB + threadIdx.x / G;
    const bool act = (p < v.npat) && (r < R);
    double d[4] = {0.0, 0.0, 0.0, 0.0};
    int m = 0;
    if (act) {
        if (op.kind == kIntInt) {
            double a[4], b[4];
            cla_load_cg<ST>(cla_ptr<ST>(v, op.c1, p, R * 4) + r * 4, a);
            cla_load_cg<ST>(cla_ptr<ST>(v, op.c2, p, R * 4) + r * 4, b);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                double L = (R == 4) ? dot4_pair(PL + 4 * i, a) : dot4_seq(PL + 4 * i, a);
                double Rr = (R == 4) ? dot4_pair(PR + 4 * i, b) : dot4_seq(PR + 4 * i, b);
                d[i] = mul(L, Rr);
            }
            if (r == 0)
                m = __ldcg(v.scalers + (long long)op.c1 * v.npat_pad + p) + __ldcg(v.scalers + (long long)op.c2 * v.npat_pad + p);
        } else if (op.kind == kIntTip) {
            double a[4];
            cla_load_cg<ST>(cla_ptr<ST>(v, op.c1, p, R * 4) + r * 4, a);
            const int code = v.tips[(long long)op.c2 * v.npat_pad + p];
            const int cls = tip_class(code);
            if (cls == 0) {
                const int s = __ffs(code & 15) - 1;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    double L = (R == 4) ? dot4_pair(PL + 4 * i, a) : dot4_seq(PL + 4 * i, a);
                    const double pr = s == 0 ? PR[4 * i] : s == 1 ? PR[4 * i + 1] : s == 2 ? PR[4 * i + 2] : PR[4 * i + 3];
                    d[i] = mul(L, pr);
                }
            } else if (cls == 1) {
#pragma unroll
                for (int i = 0; i < 4; i++) d[i] = dot4_seq(PL + 4 * i, a);
            } else {
                double tv[4];
                tip_vec(PR, code, tv);
#pragma unroll
                for (int i = 0; i < 4; i++) d[i] = mul(tv[i], dot4_seq(PL + 4 * i, a));
            }
            if (r == 0) m = __ldcg(v.scalers + (long long)op.c1 * v.npat_pad + p);
        } else {
            double tl[4], tr[4];
            tip_vec(PL, v.tips[(long long)op.c1 * v.npat_pad + p], tl);
            tip_vec(PR, v.tips[(long long)op.c2 * v.npat_pad + p], tr);
#pragma unroll
            for (int i = 0; i < 4; i++) d[i] = mul(tl[i], tr[i]);
        }
    }
    if (GARLI_SCALE) {
        if (op.rescale) {
            double mx = act ? fmax(fmax(d[0], d[2]), fmax(d[1], d[3])) : 0.0;
#pragma unroll
            for (int o = 1; o < G; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (act && mx < c_rescale_below) {
                if (mx < c_reduce_below && (v.rescale_every > 2 || mx < c_bail_below)) {
                    if (r == 0) atomicOr(v.status, kStatusRescaleRetry);
                }
                int idx = 0;
                while ((idx + 1) < kRescaleTableLen && c_thresh[idx + 1] > mx) idx++;
                const double mu = c_mult[idx];
#pragma unroll
                for (int i = 0; i < 4; i++) d[i] = mul(d[i], mu);
                m += c_incr[idx];
            }
        }
    } else {
        double mx = act ? fmax(fmax(d[0], d[2]), fmax(d[1], d[3])) : 0.0;
#pragma unroll
        for (int o = 1; o < G; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (act && mx > 0.0) {
            const int e = ilogb(mx);
            const double sc = ldexp(1.0, -e);
#pragma unroll
            for (int i = 0; i < 4; i++) d[i] *= sc;
            m -= e;
        }
    }
    if (act) {
        cla_store<ST>(cla_ptr<ST>(v, op.dest, p, R * 4) + r * 4, d);
        if (r == 0) v.scalers[(long long)op.dest * v.npat_pad + p] = m;
    }
}

struct PassArgs {
    const PCmd *cmds;
    int ncmd;
    const DevOp *ops;
    NrParams prm;
    double *lengths;
    const double *eig;
    const double *rates;
    NrSlot *slots;
    GridSync *gs;
    double *sums2;  // two partial-sum buffers of 3 * nvb doubles (double-buffered per iteration)
    int nvb;        // virtual blocks of the edge sweep (the host edge kernel's grid)
    unsigned long long *trace;  // optional phase timestamps of block 0: (code << 56) | ns
    int trace_cap;
};

enum TraceCode : int { kTrLevel = 1, kTrLevelDone, kTrNewton, kTrSweep, kTrBarrier, kTrStep, kTrNewtonDone };

template <int R, bool GARLI_SCALE>
__global__ void __launch_bounds__(kThreads) k_pass4(View v, PassArgs A) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    __shared__ EdgeSmem<R, true> sm;
    __shared__ double red[3][kThreads];
    __shared__ double pscratch[3 * R * 4];
    __shared__ NrState st;
    __shared__ int s_fin;
    const int lane_r = threadIdx.x % G;
    const int rr = lane_r < R ? lane_r : 0;
    const int ntiles = (v.npat + PPB - 1) / PPB;
    int parity = 0;
    int ntr = 0;
    auto mark = [&](int code) {
        if (A.trace && blockIdx.x == 0 && threadIdx.x == 0 && ntr < A.trace_cap)
            A.trace[ntr++] = ((unsigned long long)code << 56) | (global_ns() & ((1ULL << 56) - 1));
    };
    for (int ci = 0; ci < A.ncmd; ci++) {
        const PCmd cmd = A.cmds[ci];
        mark(cmd.type == kCmdLevel ? kTrLevel : kTrNewton);
        if (cmd.type == kCmdLevel) {
            // Pattern-local (enough 256-pattern chunks for half the blocks):
            // for every op of the level this block updates the chunks whose
            // edge sums it also takes (chunk c belongs to virtual block c mod
            // nvb, virtual block vb to block vb mod grid).  An update reads its
            // children at the same patterns and the rescale rule is per op and
            // pattern, so what it needs was written by this block: a block
            // barrier orders it, no grid barrier.  With fewer chunks the
            // level's (op, tile) items spread over every block and a grid
            // barrier ends the level.
            const int nchunks = (v.npat + kThreads - 1) / kThreads;
            if (2 * nchunks >= (int)gridDim.x) {
                for (int j = 0; j < cmd.b; j++) {
                    const DevOp op = A.ops[cmd.a + j];
                    double PL[16], PR[16];
                    const double *m1 = v.mats + (long long)op.p1 * v.mat_stride + 16 * rr;
                    const double *m2 = v.mats + (long long)op.p2 * v.mat_stride + 16 * rr;
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        PL[i] = __ldcg(m1 + i);
                        PR[i] = __ldcg(m2 + i);
                    }
                    for (int vb = blockIdx.x; vb < A.nvb; vb += gridDim.x)
                        for (int c = vb; c < nchunks; c += A.nvb)
                            for (int tile = c * G; tile < min(ntiles, (c + 1) * G); tile++)
                                cla4_tile_cg<double, R, GARLI_SCALE>(v, op, PL, PR, tile);  // FP64 throughout
                    __syncthreads();
                }
            } else {
                const long long nitems = (long long)cmd.b * ntiles;
                int cur = -1;
                double PL[16], PR[16];
                for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
                    const int j = (int)(item / ntiles), tile = (int)(item % ntiles);
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
                    cla4_tile_cg<double, R, GARLI_SCALE>(v, op, PL, PR, tile);  // plain form: FP64 throughout
                }
                if (!grid_barrier(A.gs, v.status)) return;
            }
            mark(kTrLevelDone);
        } else {
            const int pbuf = cmd.a, cbuf = cmd.b, tip = cmd.c, mat = cmd.d;
            // P at the current length is in mats[mat]; frequencies and rate weights
            {
                const double *mp = v.mats + (long long)mat * v.mat_stride;
                for (int i = threadIdx.x; i < R * 16; i += blockDim.x) {
                    sm.M[0][i] = __ldcg(mp + i);
                    sm.M[1][i] = __ldcg(mp + R * 16 + i);
                    sm.M[2][i] = __ldcg(mp + 2 * R * 16 + i);
                }
                if (threadIdx.x < 4) sm.F[threadIdx.x] = v.freqs[threadIdx.x];
                if (threadIdx.x < R) sm.RP[threadIdx.x] = v.rate_probs[threadIdx.x];
                if (threadIdx.x == 0) nr_init(st, __ldcg(A.lengths + mat), A.prm.min_brlen, A.prm.max_brlen);
            }
            __syncthreads();
            int evals = 0;
            double last_lnL = 0.0, last_d1 = 0.0, last_d2 = 0.0;
            for (;;) {
                double *sums = A.sums2 + (long long)parity * 3 * A.nvb;
                parity ^= 1;
                for (int vb = blockIdx.x; vb < A.nvb; vb += gridDim.x) {
                    double aL = 0.0, a1 = 0.0, a2 = 0.0;
                    for (int p = vb * kThreads + threadIdx.x; p < v.npat; p += A.nvb * kThreads) {
                        edge4_site_cg<double, R, GARLI_SCALE>(v, sm, pbuf, cbuf, tip, p, aL, a1, a2);
                    }
                    block_sum3(aL, a1, a2, sums + 3 * vb);
                    __syncthreads();
                }
                mark(kTrSweep);
                if (!grid_barrier(A.gs, v.status)) return;
                mark(kTrBarrier);
                // every block: the k_reduce3 reduction of all partial sums
                {
                    double a = 0.0, b = 0.0, c = 0.0;
                    for (int i = threadIdx.x; i < A.nvb; i += blockDim.x) {
                        a += __ldcg(sums + 3 * i);
                        b += __ldcg(sums + 3 * i + 1);
                        c += __ldcg(sums + 3 * i + 2);
                    }
                    red[0][threadIdx.x] = a;
                    red[1][threadIdx.x] = b;
                    red[2][threadIdx.x] = c;
                    __syncthreads();
                    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
                        if ((int)threadIdx.x < w) {
                            red[0][threadIdx.x] += red[0][threadIdx.x + w];
                            red[1][threadIdx.x] += red[1][threadIdx.x + w];
                            red[2][threadIdx.x] += red[2][threadIdx.x + w];
                        }
                        __syncthreads();
                    }
                }
                if (threadIdx.x == 0) {
                    last_lnL = red[0][0];
                    last_d1 = red[1][0];
                    last_d2 = red[2][0];
                    s_fin = nr_step(st, last_d1, last_d2, last_lnL, A.prm.precision, A.prm.min_brlen, A.prm.max_brlen);
                }
                evals++;
                __syncthreads();
                pmat4_smem<R>(A.eig, A.rates, v.pinv, v.has_pinv, st.v, sm.M, pscratch);
                mark(kTrStep);
                if (s_fin) break;
            }
            // The branch's final length and P for the CLA updates that follow.
            // Every block took the same steps from the same sums and holds the
            // same P: each writes it (identical values) and reads back its own
            // copy in the levels that follow -- no grid barrier.
            {
                double *mp = const_cast<double *>(v.mats) + (long long)mat * v.mat_stride;
                for (int i = threadIdx.x; i < R * 16; i += blockDim.x) {
                    mp[i] = sm.M[0][i];
                    mp[R * 16 + i] = sm.M[1][i];
                    mp[2 * R * 16 + i] = sm.M[2][i];
                }
                if (blockIdx.x == 0 && threadIdx.x == 0) {
                    A.lengths[mat] = st.v;
                    NrSlot &sl = A.slots[mat];
                    sl.st = st;
                    sl.lnL = last_lnL;
                    sl.d1 = last_d1;
                    sl.d2 = last_d2;
                    sl.evals = evals;
                }
            }
            __syncthreads();
            mark(kTrNewtonDone);
        }
    }
}

}  // namespace gb
