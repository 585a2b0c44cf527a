// gb_nstate.cuh -- 20-state (amino acid) and 61-state (codon) kernels.
//
// CUDA-core FP64 versions that keep GARLI's per-site arithmetic order
// (sequential sums over "to" states, tree.cpp:7843-7910, :8537-8600,
// :5597-6460, optimization.cpp:2592-3614).  A block owns a tile of TP
// patterns; the two P(t) sets of the op and the children's tiles are staged
// in shared memory, each thread produces (pattern, from-state) outputs, and
// the tile of results stays in shared memory until the per-pattern rescale
// decision has been taken.
#pragma once
#include "gb_common.cuh"
#include "gb_dna.cuh"

namespace gb {

template <typename ST>
__device__ __forceinline__ double ldv(const ST *p) { return (double)__ldg(p); }

// copy n consecutive CLA values of buffer b starting at pattern p0 into shared memory
__device__ __forceinline__ void tile_load(const View &v, int b, int p0, int RS, int n, double *dst) {
    if (p0 < v.kpad) {
        const double *src = cla_ptr<double>(v, b, p0, RS);
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = ldv<double>(src + i);
    } else {
        const float *src = cla_ptr<float>(v, b, p0, RS);
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = ldv<float>(src + i);
    }
}

// dynamic shared memory layout for k_cla_ns:
//   PL[R*S*S], PR[R*S*S], A[TP*R*S], B[TP*R*S], D[TP*R*S], mx[TP], mlt[TP]
// P is held transposed, [rate][to][from]: the threads of a warp take
// consecutive "from" states, so each "to" step reads consecutive words
// (P's rows are S doubles apart: read by rows, 20 states put 8 threads on a bank).
template <bool GARLI_SCALE>
__global__ void __launch_bounds__(kThreads) k_cla_ns(View v, LevelOps ops, int S, int R, int TP) {
    extern __shared__ double sm[];
    const DevOp op = ops.op[blockIdx.y];
    const int RS = R * S, RSS = R * S * S, SS = S * S;
    double *PL = sm, *PR = PL + RSS, *A = PR + RSS, *B = A + TP * RS, *D = B + TP * RS;
    double *mx = D + TP * RS;
    const double *m1 = v.mats + (long long)op.p1 * v.mat_stride;
    const double *m2 = v.mats + (long long)op.p2 * v.mat_stride;
    for (int i = threadIdx.x; i < RSS; i += blockDim.x) {
        const int r = i / SS, from = (i % SS) / S, to = i % S;
        PL[r * SS + to * S + from] = m1[i];
        PR[r * SS + to * S + from] = m2[i];
    }
    const int p0 = blockIdx.x * TP;
    const int np = min(TP, v.npat - p0);
    if (op.kind != kTipTip) tile_load(v, op.c1, p0, RS, np * RS, A);
    if (op.kind == kIntInt) tile_load(v, op.c2, p0, RS, np * RS, B);
    __syncthreads();
    for (int o = threadIdx.x; o < np * RS; o += blockDim.x) {
        const int pl = o / RS, rem = o % RS, r = rem / S, from = rem % S;
        const int p = p0 + pl;
        // P[from][to] of this rate is pl_col[to * S]
        const double *pl_col = PL + r * SS + from;
        const double *pr_col = PR + r * SS + from;
        double val;
        if (op.kind == kIntInt) {
            const double *a = A + pl * RS + r * S, *b = B + pl * RS + r * S;
            double L1 = 0.0, R1 = 0.0;
            for (int to = 0; to < S; to++) {
                L1 = add(L1, mul(pl_col[to * S], a[to]));
                R1 = add(R1, mul(pr_col[to * S], b[to]));
            }
            val = mul(L1, R1);
        } else if (op.kind == kIntTip) {
            const double *a = A + pl * RS + r * S;
            double acc = 0.0;
            for (int to = 0; to < S; to++) acc = add(acc, mul(pl_col[to * S], a[to]));
            const int s2 = v.tips[(long long)op.c2 * v.npat_pad + p];
            val = (s2 < S) ? mul(acc, pr_col[s2 * S]) : acc;
        } else {
            const int l = v.tips[(long long)op.c1 * v.npat_pad + p];
            const int rr = v.tips[(long long)op.c2 * v.npat_pad + p];
            const double tl = (l < S) ? pl_col[l * S] : 1.0;
            const double tr = (rr < S) ? pr_col[rr * S] : 1.0;
            val = mul(tl, tr);
        }
        D[o] = val;
    }
    __syncthreads();
    // per-pattern largest entry (RescaleRateHetNState, tree.cpp:3492-3598)
    for (int pl = threadIdx.x; pl < np; pl += blockDim.x) {
        double large = D[pl * RS] > D[pl * RS + 1] ? D[pl * RS] : D[pl * RS + 1];
        for (int s = 2; s < RS; s++) large = D[pl * RS + s] > large ? D[pl * RS + s] : large;
        const int p = p0 + pl;
        int m = 0;
        if (op.kind == kIntInt) m = v.scalers[(long long)op.c1 * v.npat_pad + p] + v.scalers[(long long)op.c2 * v.npat_pad + p];
        else if (op.kind == kIntTip) m = v.scalers[(long long)op.c1 * v.npat_pad + p];
        double mult = 1.0;
        if (GARLI_SCALE) {
            if (op.rescale && large < c_rescale_below) {
                if (large < c_reduce_below && (v.rescale_every > 2 || large < c_bail_below))
                    atomicOr(v.status, kStatusRescaleRetry);
                int idx = 0;
                while ((idx + 1) < kRescaleTableLen && c_thresh[idx + 1] > large) idx++;
                mult = c_mult[idx];
                m += c_incr[idx];
            }
        } else if (large > 0.0) {
            const int e = ilogb(large);
            mult = ldexp(1.0, -e);
            m -= e;
        }
        mx[pl] = mult;
        v.scalers[(long long)op.dest * v.npat_pad + p] = m;
    }
    __syncthreads();
    if (p0 < v.kpad) {
        double *dst = cla_ptr<double>(v, op.dest, p0, RS);
        for (int o = threadIdx.x; o < np * RS; o += blockDim.x) {
            const double mult = mx[o / RS];
            dst[o] = mult != 1.0 ? mul(D[o], mult) : D[o];
        }
    } else {
        float *dst = cla_ptr<float>(v, op.dest, p0, RS);
        for (int o = threadIdx.x; o < np * RS; o += blockDim.x) {
            const double mult = mx[o / RS];
            // keyed on the value's offset in the CLA pool: the same rounding in every run
            const unsigned int key = (unsigned int)((reinterpret_cast<const char *>(dst + o) - v.partials) >> 2);
            dst[o] = round_stochastic(mult != 1.0 ? mul(D[o], mult) : D[o], key);
        }
    }
}

// Edge evaluation for S states: per-(pattern, rate, from) terms computed in
// parallel, then summed per pattern in the reference's order.
// dynamic smem: M[3*R*S*S], C[TP*R*S], Pp[TP*R*S], T[3*TP*R*S], freqs[S], rp[R]
template <bool GARLI_SCALE, bool DERIV>
__global__ void __launch_bounds__(kThreads) k_edge_ns(View v, int pbuf, int cbuf, int mat, int child_tip,
                                                      int write_sites, int S, int R, int TP) {
    extern __shared__ double sm[];
    const int RS = R * S, RSS = R * S * S, SS = S * S;
    double *M = sm, *C = M + 3 * RSS, *Pp = C + TP * RS, *T = Pp + TP * RS, *F = T + 3 * TP * RS, *RP = F + S;
    const double *mp = v.mats + (long long)mat * v.mat_stride;
    // P, dP, d2P transposed, [matrix][rate][to][from] (as in k_cla_ns)
    for (int i = threadIdx.x; i < (DERIV ? 3 : 1) * RSS; i += blockDim.x) {
        const int k = i / RSS, j = i % RSS, r = j / SS, from = (j % SS) / S, to = j % S;
        M[k * RSS + r * SS + to * S + from] = mp[i];
    }
    for (int i = threadIdx.x; i < S; i += blockDim.x) F[i] = v.freqs[i];
    for (int i = threadIdx.x; i < R; i += blockDim.x) RP[i] = v.rate_probs[i];
    double accL = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int p0 = blockIdx.x * TP; p0 < v.npat; p0 += gridDim.x * TP) {
        const int np = min(TP, v.npat - p0);
        __syncthreads();
        tile_load(v, pbuf, p0, RS, np * RS, Pp);
        if (!child_tip) tile_load(v, cbuf, p0, RS, np * RS, C);
        __syncthreads();
        for (int o = threadIdx.x; o < np * RS; o += blockDim.x) {
            const int pl = o / RS, rem = o % RS, r = rem / S, from = rem % S;
            const int p = p0 + pl;
            const double *col = M + r * SS + from;  // P[from][to] = col[to * S]
            double l = 0.0, a = 0.0, b = 0.0;
            if (!child_tip) {
                const double *c = C + pl * RS + r * S;
                for (int to = 0; to < S; to++) {
                    l = add(l, mul(col[to * S], c[to]));
                    if (DERIV) {
                        a = add(a, mul(col[RSS + to * S], c[to]));
                        b = add(b, mul(col[2 * RSS + to * S], c[to]));
                    }
                }
            } else {
                const int s = v.tips[(long long)cbuf * v.npat_pad + p];
                if (s < S) {
                    l = col[s * S];
                    if (DERIV) {
                        a = col[RSS + s * S];
                        b = col[2 * RSS + s * S];
                    }
                } else {
                    l = 1.0;  // total ambiguity: partial*freq only, no derivative terms
                }
            }
            const double w = Pp[pl * RS + r * S + from];
            const bool amb = child_tip && v.tips[(long long)cbuf * v.npat_pad + p] >= S;
            // reference: temp * partial[from] * freqs[from]  (ambiguous tip: partial[from] * freqs[from])
            T[o] = amb ? mul(w, F[from]) : mul(mul(l, w), F[from]);
            if (DERIV) {
                T[TP * RS + o] = mul(mul(a, w), F[from]);
                T[2 * TP * RS + o] = mul(mul(b, w), F[from]);
            }
        }
        __syncthreads();
        for (int pl = threadIdx.x; pl < np; pl += blockDim.x) {
            const int p = p0 + pl;
            double siteL = 0.0, sD1 = 0.0, sD2 = 0.0;
            if (R == 1) {
                for (int from = 0; from < S; from++) {
                    siteL = add(siteL, T[pl * RS + from]);
                    if (DERIV) {
                        sD1 = add(sD1, T[TP * RS + pl * RS + from]);
                        sD2 = add(sD2, T[2 * TP * RS + pl * RS + from]);
                    }
                }
                siteL = mul(siteL, RP[0]);
                if (DERIV) {
                    sD1 = mul(sD1, RP[0]);
                    sD2 = mul(sD2, RP[0]);
                }
            } else {
                for (int r = 0; r < R; r++) {
                    double rL = 0.0, r1 = 0.0, r2 = 0.0;
                    for (int from = 0; from < S; from++) {
                        rL = add(rL, T[pl * RS + r * S + from]);
                        if (DERIV) {
                            r1 = add(r1, T[TP * RS + pl * RS + r * S + from]);
                            r2 = add(r2, T[2 * TP * RS + pl * RS + r * S + from]);
                        }
                    }
                    siteL = add(siteL, mul(rL, RP[r]));
                    if (DERIV) {
                        sD1 = add(sD1, mul(r1, RP[r]));
                        sD2 = add(sD2, mul(r2, RP[r]));
                    }
                }
            }
            const int m1 = v.scalers[(long long)pbuf * v.npat_pad + p];
            const int m2 = child_tip ? 0 : v.scalers[(long long)cbuf * v.npat_pad + p];
            if (v.has_pinv && v.const_states[p] >= 0) {
                const double pf = mul(v.pinv, F[v.const_states[p]]);
                if (GARLI_SCALE) {
                    if (DERIV) {
                        // prI*freq*exp(partial)*exp(child) (optimization.cpp:3300, :3507)
                        siteL = child_tip ? add(siteL, mul(pf, exp((double)m1)))
                                          : add(siteL, mul(mul(pf, exp((double)m1)), exp((double)m2)));
                    } else if (m1 + m2 == 0) {
                        siteL = add(siteL, pf);
                    } else {
                        siteL = add(siteL, mul(pf, exp(add((double)m1, (double)m2))));
                    }
                } else {
                    siteL = add(siteL, ldexp(pf, m1 + m2));
                }
            }
            double u;
            if (GARLI_SCALE) u = sub(sub(log(siteL), (double)m1), (double)m2);
            else u = sub(log(siteL), (double)(m1 + m2) * 0.69314718055994530941723212145818);
            if (write_sites) v.site_lnl[p] = u;
            double d1 = 0.0, d2 = 0.0;
            if (DERIV) {
                d1 = sD1 / siteL;
                d2 = sub(sD2 / siteL, mul(d1, d1));
                if (write_sites) {
                    v.site_d1[p] = d1;
                    v.site_d2[p] = d2;
                }
            }
            // GARLI drops non-negative site lnLs (tree.cpp:6380, optimization.cpp:3378)
            if (u < 0.0) {
                const double cnt = (double)v.counts[p];
                accL = add(accL, mul(u, cnt));
                if (DERIV) {
                    acc1 = add(acc1, mul(cnt, d1));
                    acc2 = add(acc2, mul(cnt, d2));
                }
            }
        }
    }
    __syncthreads();
    block_sum3(accL, acc1, acc2, v.block_sums + 3 * blockIdx.x);
}

}  // namespace gb
