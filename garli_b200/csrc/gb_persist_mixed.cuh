// gb_persist_mixed.cuh -- the single-tree persistent pass of the precision form.
//
// Same device command queue and Newton scheme as k_pass4 (gb_persist.cuh):
// levels of CLA updates and, per branch, Newton-Raphson iterations in which
// every block sums lnL/d1/d2 over its share of the patterns, one grid
// barrier, then every block reduces all partial sums in the same fixed order
// and takes the same gb::nr_step.  The precision form differs in its
// arithmetic, not its decisions' structure:
//   * CLA levels use the batched kernel's code (cla_tiles_m): one lane per
//     (pattern, category), the op's P blocks in shared memory, FP64 fused
//     arithmetic, both children's loads issued before any arithmetic,
//     compact stores; each block updates the patterns whose edge sums it
//     takes, so levels and branch ends need no grid barrier -- only the
//     Newton sums do;
//   * the edge sweep loads the partial and child slices of all categories
//     first and evaluates P, dP, d2P with fused FP64 multiply-adds.
#pragma once
#include "gb_batch_mixed.cuh"
#include "gb_persist.cuh"

namespace gb {

// lnL, d1, d2 of pattern p across the branch (GetScorePartial*RateHet,
// tree.cpp:6040/:6172; GetDerivsPartial*, optimization.cpp:2412/:3063), fused FP64
template <int R>
__device__ __forceinline__ void edge4m_site(const View &v, const EdgeSmem<R, true> &sm, int pbuf, int cbuf,
                                            int child_tip, int p, double &accL, double &acc1, double &acc2) {
    const double *f = sm.F;
    double part[R][4], ch[R][4];
#pragma unroll
    for (int r = 0; r < R; r++) {
        slice_load<R>(v, pbuf, false, p, r, part[r]);
        if (!child_tip) slice_load<R>(v, cbuf, false, p, r, ch[r]);
    }
    const int m1 = __ldcg(v.scalers + (long long)pbuf * v.npat_pad + p);
    const int m2 = child_tip ? 0 : __ldcg(v.scalers + (long long)cbuf * v.npat_pad + p);
    double L[4] = {0, 0, 0, 0}, D1[4] = {0, 0, 0, 0}, D2[4] = {0, 0, 0, 0};
    if (!child_tip) {
#pragma unroll
        for (int r = 0; r < R; r++) {
            double t0[4], t1[4], t2[4];
            pvec(&sm.M[0][16 * r], ch[r], t0);
            pvec(&sm.M[1][16 * r], ch[r], t1);
            pvec(&sm.M[2][16 * r], ch[r], t2);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double w = part[r][i] * sm.RP[r];
                L[i] = fma(t0[i], w, L[i]);
                D1[i] = fma(t1[i], w, D1[i]);
                D2[i] = fma(t2[i], w, D2[i]);
            }
        }
    } else {
        const int code = v.tips[(long long)cbuf * v.npat_pad + p] & 15;
        if (code == 15 || code == 0) {
            // total ambiguity: the partial weighted by the category probabilities
#pragma unroll
            for (int r = 0; r < R; r++)
#pragma unroll
                for (int i = 0; i < 4; i++) L[i] = fma(part[r][i], sm.RP[r], L[i]);
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) {
                double t0[4], t1[4], t2[4];
                pvec_tip(&sm.M[0][16 * r], code, t0);
                pvec_tip(&sm.M[1][16 * r], code, t1);
                pvec_tip(&sm.M[2][16 * r], code, t2);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const double w = part[r][i] * sm.RP[r];
                    L[i] = fma(t0[i], w, L[i]);
                    D1[i] = fma(t1[i], w, D1[i]);
                    D2[i] = fma(t2[i], w, D2[i]);
                }
            }
        }
    }
    double siteL = fma(L[3], f[3], fma(L[2], f[2], fma(L[1], f[1], L[0] * f[0])));
    const int cb = v.const_states[p];
    if (v.has_pinv && cb >= 0) {
        double btot = 0.0;
#pragma unroll
        for (int s = 0; s < 4; s++)
            if (cb & (1 << s)) btot += f[s];
        siteL += ldexp(v.pinv * btot, m1 + m2);
    }
    const double cnt = (double)v.counts[p];
    const double inv = 1.0 / siteL;
    const double sd1 = fma(D1[3], f[3], fma(D1[2], f[2], fma(D1[1], f[1], D1[0] * f[0]))) * inv;
    const double sd2 = fma(fma(D2[3], f[3], fma(D2[2], f[2], fma(D2[1], f[1], D2[0] * f[0]))), inv, -sd1 * sd1);
    accL = fma(cnt, log(siteL) - (double)(m1 + m2) * 0.69314718055994530941723212145818, accL);
    acc1 = fma(cnt, sd1, acc1);
    acc2 = fma(cnt, sd2, acc2);
}

template <int R>
__global__ void __launch_bounds__(kThreads, 2) k_pass4m(View v, PassArgs A) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    __shared__ EdgeSmem<R, true> sm;
    __shared__ double red[3][kThreads / 32];
    __shared__ double pscratch[3 * R * 4];
    __shared__ __align__(16) double sP[2][R][kPStride];
    __shared__ NrState st;
    __shared__ int s_fin;
    const int cr = threadIdx.x % G;
    const bool cla_ok = cr < R;
    const int crr = cla_ok ? cr : 0;
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
            // children at the same patterns, so what it needs was written by
            // this block: a block barrier orders it, no grid barrier.  With
            // fewer chunks the level's (op, tile pair) items spread over every
            // block and a grid barrier ends the level.
            const int nchunks = (v.npat + kThreads - 1) / kThreads;
            if (2 * nchunks >= (int)gridDim.x) {
                for (int j = 0; j < cmd.b; j++) {
                    const DevOp op = A.ops[cmd.a + j];
                    __syncthreads();
                    for (int q = threadIdx.x; q < 2 * R * 16; q += blockDim.x) {
                        const int mi = q / (R * 16), rem = q % (R * 16);
                        sP[mi][rem / 16][rem % 16] =
                            __ldcg(v.mats + (long long)(mi ? op.p2 : op.p1) * v.mat_stride + rem);
                    }
                    __syncthreads();
                    for (int vb = blockIdx.x; vb < A.nvb; vb += gridDim.x)
                        for (int c = vb; c < nchunks; c += A.nvb)
                            cla_tiles_m<R>(v, op, sP[0][crr], sP[1][crr], c * G, min(ntiles, (c + 1) * G), crr,
                                           cla_ok);
                }
                __syncthreads();
            } else {
                const int items_per_op = (ntiles + 1) / 2;
                const long long nitems = (long long)cmd.b * items_per_op;
                int cur = -1;
                DevOp op;
                for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
                    const int j = (int)(item / items_per_op);
                    const int t0 = (int)(item % items_per_op) * 2;
                    if (j != cur) {  // uniform across the block
                        cur = j;
                        op = A.ops[cmd.a + j];
                        __syncthreads();
                        for (int q = threadIdx.x; q < 2 * R * 16; q += blockDim.x) {
                            const int mi = q / (R * 16), rem = q % (R * 16);
                            sP[mi][rem / 16][rem % 16] =
                                __ldcg(v.mats + (long long)(mi ? op.p2 : op.p1) * v.mat_stride + rem);
                        }
                        __syncthreads();
                    }
                    cla_tiles_m<R>(v, op, sP[0][crr], sP[1][crr], t0, min(ntiles, t0 + 2), crr, cla_ok);
                }
                if (!grid_barrier(A.gs, v.status)) return;
            }
            mark(kTrLevelDone);
            continue;
        }
        const int pbuf = cmd.a, cbuf = cmd.b, tip = cmd.c, mat = cmd.d;
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
                for (int p = vb * kThreads + threadIdx.x; p < v.npat; p += A.nvb * kThreads)
                    edge4m_site<R>(v, sm, pbuf, cbuf, tip, p, aL, a1, a2);
                block_sum3(aL, a1, a2, sums + 3 * vb);
                __syncthreads();
            }
            mark(kTrSweep);
            if (!grid_barrier(A.gs, v.status)) return;
            mark(kTrBarrier);
            {
                // every block: the same fixed-order sum of all partial sums
                // (strided per thread, shuffle tree per warp, warps in order)
                double a = 0.0, b = 0.0, c = 0.0;
                for (int i = threadIdx.x; i < A.nvb; i += blockDim.x) {
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
                if ((threadIdx.x & 31) == 0) {
                    red[0][threadIdx.x >> 5] = a;
                    red[1][threadIdx.x >> 5] = b;
                    red[2][threadIdx.x >> 5] = c;
                }
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                last_lnL = last_d1 = last_d2 = 0.0;
                for (int w = 0; w < kThreads / 32; w++) {
                    last_lnL += red[0][w];
                    last_d1 += red[1][w];
                    last_d2 += red[2][w];
                }
                s_fin = nr_step(st, last_d1, last_d2, last_lnL, A.prm.precision, A.prm.min_brlen, A.prm.max_brlen);
            }
            evals++;
            __syncthreads();
            pmat4_smem<R>(A.eig, A.rates, v.pinv, v.has_pinv, st.v, sm.M, pscratch);
            mark(kTrStep);
            if (s_fin) break;
        }
        // Every block took the same steps from the same sums, so every block
        // holds the same optimised P: each writes it (identical values) and
        // reads back its own copy in the levels that follow -- no grid barrier.
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

}  // namespace gb
