// gb_nstate.cuh -- 20-state (amino acid) and 61-state (codon) kernels.
//
// CUDA-core FP64 versions that keep GARLI's per-site arithmetic order
// (sequential sums over "to" states, tree.cpp:7843-7910, :8537-8600,
// :5597-6460, optimization.cpp:2592-3614).  CLA updates: a block stages the
// op's two P(t) sets in shared memory once and walks pattern tiles, the next
// tile's inputs arriving by cp.async while a register tile per lane (several
// patterns x several from-states) is computed.  Edge evaluations: a block
// owns a tile of patterns, one (pattern, rate, from) term per thread, summed
// per pattern in the reference's order.
#pragma once
#include "gb_common.cuh"
#include "gb_dna.cuh"
#include "gb_stage.cuh"

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

// Register tile of the n-state CLA kernel: the 32 lanes of a warp are NF
// "from"-state groups x NQ pattern groups; a lane computes F from-states
// (fg, fg + NF, ...) of Q patterns (qg, qg + NQ, ...) of one rate category, so
// each P entry read from shared memory serves Q patterns and each child value
// serves F from-states.
template <int S>
struct NsTile {
    static constexpr int NF = S <= 20 ? 4 : 8;
    static constexpr int F = (S + NF - 1) / NF;
    static constexpr int NQ = 32 / NF;
    static constexpr int Q = 2;
    static constexpr int PW = NQ * Q;  // patterns of one warp task; tiles are multiples of it
};

// Row stride (in doubles) of a pattern in a child tile: >= RS and 2 mod 4,
// so rows start 16-byte aligned and the 16-byte reads of one "to" pair by the
// pattern groups of a warp fall in distinct banks.
__host__ __device__ inline int ns_row_stride(int RS) { return RS + (6 - RS % 4) % 4; }

// dynamic shared memory of k_cla_ns in bytes: P sets, two stages of both
// children's tiles, per-(rate, pattern) maxima and multipliers, then per
// stage the children's scalers and tip codes
__host__ __device__ inline size_t ns_cla_smem_bytes(int S, int R, int TP) {
    const size_t RS = (size_t)R * S, RSP = (size_t)ns_row_stride(R * S);
    const size_t dbl = 2 * RS * S + 4 * (size_t)TP * RSP + (size_t)R * TP + TP;
    return (dbl * 8 + 15) / 16 * 16 + 2 * 2 * (size_t)TP * 4 + 2 * 2 * (size_t)TP;
}

__device__ __forceinline__ void cp8(uint32_t dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}

// Asynchronous copy of one tile's inputs into a stage: the children's np
// patterns x RS values pattern-major in rows of RSP doubles (FP64 tiles in
// 16-byte pieces when RS is even; FP32 tiles, to be widened after the wait,
// as 16-byte pieces of floats in the tail of each row's slot when RS is a
// multiple of 4, else each value as a float in the first half of its slot),
// their
// scalers (sc[0..TP) child 1, sc[TP..2TP) child 2) and tip codes (tt[0..TP)
// child 1, tt[TP..2TP) child 2).
__device__ __forceinline__ void ns_prefetch(const View &v, const DevOp &op, int p0, int np, int RS, int RSP, int TP,
                                            double *A, double *B, int *sc, uint8_t *tt) {
    const bool dbl = p0 < v.kpad;
    for (int c = 0; c < 2; c++) {
        const bool has_cla = c == 0 ? op.kind != kTipTip : op.kind == kIntInt;
        const int buf = c == 0 ? op.c1 : op.c2;
        if (has_cla) {
            double *dst = c == 0 ? A : B;
            if (dbl && RS % 2 == 0) {
                const int H = RS / 2, n = np * H, dpl = blockDim.x / H, dh = blockDim.x % H;
                const double *src = cla_ptr<double>(v, buf, p0, RS);
                int pl = threadIdx.x / H, h = threadIdx.x % H;
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    cp16(smem_u32(dst + pl * RSP + 2 * h), src + 2 * i);
                    pl += dpl;
                    h += dh;
                    if (h >= H) { h -= H; pl++; }
                }
            } else if (!dbl && RS % 4 == 0) {
                // FP32 rows in 16-byte pieces into the tail of each row's slot (ns_widen_rows)
                const int Q4 = RS / 4, n = np * Q4, dpl = blockDim.x / Q4, dq = blockDim.x % Q4;
                const float *src = cla_ptr<float>(v, buf, p0, RS);
                const int tail = (RSP * 8 - RS * 4);
                int pl = threadIdx.x / Q4, q = threadIdx.x % Q4;
                for (int i = threadIdx.x; i < n; i += blockDim.x) {
                    cp16(smem_u32(reinterpret_cast<char *>(dst + pl * RSP) + tail + 16 * q), src + 4 * i);
                    pl += dpl;
                    q += dq;
                    if (q >= Q4) { q -= Q4; pl++; }
                }
            } else {
                const int n = np * RS, dpl = blockDim.x / RS, drs = blockDim.x % RS;
                int pl = threadIdx.x / RS, rs = threadIdx.x % RS;
                if (dbl) {
                    const double *src = cla_ptr<double>(v, buf, p0, RS);
                    for (int i = threadIdx.x; i < n; i += blockDim.x) {
                        cp8(smem_u32(dst + pl * RSP + rs), src + i);
                        pl += dpl;
                        rs += drs;
                        if (rs >= RS) { rs -= RS; pl++; }
                    }
                } else {
                    const float *src = cla_ptr<float>(v, buf, p0, RS);
                    for (int i = threadIdx.x; i < n; i += blockDim.x) {
                        cp4(smem_u32(dst + pl * RSP + rs), src + i);
                        pl += dpl;
                        rs += drs;
                        if (rs >= RS) { rs -= RS; pl++; }
                    }
                }
            }
            const int *ssrc = v.scalers + (long long)buf * v.npat_pad + p0;
            for (int q = threadIdx.x; q < np; q += blockDim.x) cp4(smem_u32(sc + c * TP + q), ssrc + q);
        } else {
            // a tip child: its codes for the whole tile (inside the padded pattern range)
            const uint8_t *tsrc = v.tips + (long long)buf * v.npat_pad + p0;
            for (int q = threadIdx.x; q < TP / 4; q += blockDim.x) cp4(smem_u32(tt + c * TP + 4 * q), tsrc + 4 * q);
        }
    }
}

// Widen an FP32 tile copied row-wise (RS a multiple of 4, at most 256): a
// warp per row reads the row's floats from the tail of its slot, then writes
// the doubles from the slot's start (all reads of the row before any write).
__device__ __forceinline__ void ns_widen_rows(const DevOp &op, int np, int RS, int RSP, double *A, double *B) {
    const int lane = threadIdx.x & 31, Q4 = RS / 4, tail = RSP * 8 - RS * 4;
    for (int c = 0; c < (op.kind == kIntInt ? 2 : op.kind == kIntTip ? 1 : 0); c++) {
        double *X = c == 0 ? A : B;
        for (int pl = threadIdx.x >> 5; pl < np; pl += blockDim.x >> 5) {
            double *row = X + pl * RSP;
            const float4 *f = reinterpret_cast<const float4 *>(reinterpret_cast<const char *>(row) + tail);
            float4 v0 = make_float4(0.f, 0.f, 0.f, 0.f), v1 = v0;
            if (lane < Q4) v0 = f[lane];
            if (lane + 32 < Q4) v1 = f[lane + 32];
            __syncwarp();
            double2 *d = reinterpret_cast<double2 *>(row);
            if (lane < Q4) {
                d[2 * lane] = make_double2((double)v0.x, (double)v0.y);
                d[2 * lane + 1] = make_double2((double)v0.z, (double)v0.w);
            }
            if (lane + 32 < Q4) {
                d[2 * lane + 64] = make_double2((double)v1.x, (double)v1.y);
                d[2 * lane + 65] = make_double2((double)v1.z, (double)v1.w);
            }
            __syncwarp();
        }
    }
}

// Widen the FP32 values this thread copied by ns_prefetch element-wise (RS
// not a multiple of 4; after its wait): the same slots, in place.
__device__ __forceinline__ void ns_widen(const DevOp &op, int np, int RS, int RSP, double *A, double *B) {
    const int n = np * RS, dpl = blockDim.x / RS, drs = blockDim.x % RS;
    for (int c = 0; c < (op.kind == kIntInt ? 2 : op.kind == kIntTip ? 1 : 0); c++) {
        double *dst = c == 0 ? A : B;
        int pl = threadIdx.x / RS, rs = threadIdx.x % RS;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double *e = dst + pl * RSP + rs;
            // IEEE float -> double on the bit fields (exact); zero and subnormals converted
            const unsigned int u = *reinterpret_cast<const unsigned int *>(e);
            const unsigned int E = (u >> 23) & 0xffu;
            *e = (E != 0u && E != 255u)
                     ? __longlong_as_double((long long)(((unsigned long long)(u >> 31) << 63) |
                                                        ((unsigned long long)(E + 896u) << 52) |
                                                        ((unsigned long long)(u & 0x7fffffu) << 29)))
                     : (double)__uint_as_float(u);
            pl += dpl;
            rs += drs;
            if (rs >= RS) { rs -= RS; pl++; }
        }
    }
}

// acc + p * a: GARLI's separate product and sum (plain form), or one fused
// multiply-add (precision form: its FP32 storage error, 2^-24, dwarfs the
// difference)
template <bool FUSED>
__device__ __forceinline__ double mac(double acc, double p, double a) {
    if constexpr (FUSED) return __fma_rn(p, a, acc);
    else return add(acc, mul(p, a));
}

// One warp task: per lane the products of Q patterns x F from-states of
// rate r.  P is [from][to] (this rate's block), a child's row of pattern q
// starts at X + q * RSP (this rate's offset added).  For even S two "to"
// steps are read per 16-byte load (P rows and child rows are 16-byte aligned);
// the sums still run over "to" one term at a time.
template <int S, bool FUSED>
__device__ __forceinline__ void ns_task(const DevOp &op, const double *pl_r, const double *pr_r, const double *Ar,
                                        const double *Br, int RSP, const uint8_t *tt, int TP, const int *pl,
                                        const int *fr, double (&val)[NsTile<S>::Q][NsTile<S>::F]) {
    constexpr int F = NsTile<S>::F, Q = NsTile<S>::Q;
    const bool two = op.kind == kIntInt;
    if (op.kind != kTipTip) {
        double aL[Q][F], aR[Q][F];
#pragma unroll
        for (int j = 0; j < Q; j++)
#pragma unroll
            for (int k = 0; k < F; k++) aL[j][k] = aR[j][k] = 0.0;
        if constexpr (S % 2 == 0) {
#pragma unroll 2
            for (int to = 0; to < S; to += 2) {
                double2 pL[F], pR[F], a[Q], b[Q];
#pragma unroll
                for (int k = 0; k < F; k++) pL[k] = *reinterpret_cast<const double2 *>(pl_r + fr[k] * S + to);
#pragma unroll
                for (int j = 0; j < Q; j++) a[j] = *reinterpret_cast<const double2 *>(Ar + pl[j] * RSP + to);
#pragma unroll
                for (int j = 0; j < Q; j++)
#pragma unroll
                    for (int k = 0; k < F; k++) {
                        aL[j][k] = mac<FUSED>(aL[j][k], pL[k].x, a[j].x);
                        aL[j][k] = mac<FUSED>(aL[j][k], pL[k].y, a[j].y);
                    }
                if (two) {
#pragma unroll
                    for (int k = 0; k < F; k++) pR[k] = *reinterpret_cast<const double2 *>(pr_r + fr[k] * S + to);
#pragma unroll
                    for (int j = 0; j < Q; j++) b[j] = *reinterpret_cast<const double2 *>(Br + pl[j] * RSP + to);
#pragma unroll
                    for (int j = 0; j < Q; j++)
#pragma unroll
                        for (int k = 0; k < F; k++) {
                            aR[j][k] = mac<FUSED>(aR[j][k], pR[k].x, b[j].x);
                            aR[j][k] = mac<FUSED>(aR[j][k], pR[k].y, b[j].y);
                        }
                }
            }
        } else {
#pragma unroll 2
            for (int to = 0; to < S; to++) {
                double pL[F], pR[F], a[Q], b[Q];
#pragma unroll
                for (int k = 0; k < F; k++) pL[k] = pl_r[fr[k] * S + to];
#pragma unroll
                for (int j = 0; j < Q; j++) a[j] = Ar[pl[j] * RSP + to];
#pragma unroll
                for (int j = 0; j < Q; j++)
#pragma unroll
                    for (int k = 0; k < F; k++) aL[j][k] = mac<FUSED>(aL[j][k], pL[k], a[j]);
                if (two) {
#pragma unroll
                    for (int k = 0; k < F; k++) pR[k] = pr_r[fr[k] * S + to];
#pragma unroll
                    for (int j = 0; j < Q; j++) b[j] = Br[pl[j] * RSP + to];
#pragma unroll
                    for (int j = 0; j < Q; j++)
#pragma unroll
                        for (int k = 0; k < F; k++) aR[j][k] = mac<FUSED>(aR[j][k], pR[k], b[j]);
                }
            }
        }
        if (two) {
#pragma unroll
            for (int j = 0; j < Q; j++)
#pragma unroll
                for (int k = 0; k < F; k++) val[j][k] = mul(aL[j][k], aR[j][k]);
        } else {
#pragma unroll
            for (int j = 0; j < Q; j++) {
                const int s2 = tt[TP + pl[j]];
#pragma unroll
                for (int k = 0; k < F; k++)
                    val[j][k] = (s2 < S) ? mul(aL[j][k], pr_r[fr[k] * S + s2]) : aL[j][k];
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < Q; j++) {
            const int l = tt[pl[j]], rr = tt[TP + pl[j]];
#pragma unroll
            for (int k = 0; k < F; k++) {
                const double tl = (l < S) ? pl_r[fr[k] * S + l] : 1.0;
                const double tr = (rr < S) ? pr_r[fr[k] * S + rr] : 1.0;
                val[j][k] = mul(tl, tr);
            }
        }
    }
}

// CLA update for S states (CalcFullCLAInternalInternalNState and the
// internal-terminal / terminal-terminal forms, tree.cpp:7843-7910, :8537-8600,
// rescaled as RescaleRateHetNState, tree.cpp:3492-3598).  Every output is
// GARLI's expression in GARLI's order: per child a sequential sum over "to"
// of P[from][to] * CLA[to], then the product of the two children; without
// fused multiply-add in the plain form (GARLI_SCALE), fused in the precision
// form.  A block keeps the op's two P(t) sets in shared memory
// and walks pattern tiles of TP (grid-stride over plim patterns), two stages
// deep: the next tile's children, scalers and tip codes arrive by cp.async
// while the current one is computed.  A tile is R x TP / PW warp tasks (rate,
// PW patterns), at most one per warp; a task's products stay in registers
// until the pattern's multiplier is known, then go to the CLA.
//   shared: PL[R][S][S], PR (P as in global memory), stage 0 and 1: A[TP][RSP],
//   B[TP][RSP]; mxr[R][TP], mx[TP]; scalers [stage][child][TP] (int), tip codes
//   [stage][child][TP] (bytes)
template <bool GARLI_SCALE, int S>
__global__ void __launch_bounds__(kThreads) k_cla_ns(View v, LevelOps ops, int R, int TP, int plim) {
    using T = NsTile<S>;
    constexpr int NF = T::NF, F = T::F, NQ = T::NQ, Q = T::Q, SS = S * S;
    extern __shared__ __align__(16) double sm[];
    const DevOp op = ops.op[blockIdx.y];
    const int RS = R * S, RSS = R * SS, RSP = ns_row_stride(RS);
    double *PL = sm, *PR = PL + RSS, *stg = PR + RSS, *mxr = stg + 4 * TP * RSP, *mx = mxr + R * TP;
    char *tail = reinterpret_cast<char *>(sm) + ((size_t)(2 * RSS + 4 * TP * RSP + R * TP + TP) * 8 + 15) / 16 * 16;
    int *scs = reinterpret_cast<int *>(tail);                  // [stage][child][TP]
    uint8_t *tts = reinterpret_cast<uint8_t *>(scs + 4 * TP);  // [stage][child][TP]
    const int ntiles = (plim + TP - 1) / TP;
    if ((int)blockIdx.x >= ntiles) return;
    ns_prefetch(v, op, blockIdx.x * TP, min(TP, plim - (int)blockIdx.x * TP), RS, RSP, TP, stg, stg + TP * RSP, scs,
                tts);
    cp_commit();
    const double *m1 = v.mats + (long long)op.p1 * v.mat_stride;
    const double *m2 = v.mats + (long long)op.p2 * v.mat_stride;
    for (int i = threadIdx.x; i < RSS; i += blockDim.x) {
        PL[i] = m1[i];
        PR[i] = m2[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int fg = lane % NF, qg = lane / NF;
    const int tasks = R * (TP / T::PW);  // <= warps of the block (host-chosen TP)
    const bool worker = warp < tasks;
    const int r = worker ? warp % R : 0, pb = worker ? (warp / R) * T::PW : 0;
    int fr[F], pl[Q];
#pragma unroll
    for (int k = 0; k < F; k++) fr[k] = min(fg + NF * k, S - 1);  // lanes past S compute a copy, store nothing
#pragma unroll
    for (int j = 0; j < Q; j++) pl[j] = pb + qg + NQ * j;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int st = it & 1;
        const int p0 = tile * TP, np = min(TP, plim - p0);
        double *A = stg + st * 2 * TP * RSP, *B = A + TP * RSP;
        const int *sc = scs + st * 2 * TP;
        const uint8_t *tt = tts + st * 2 * TP;
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) {
            double *An = stg + (st ^ 1) * 2 * TP * RSP;
            ns_prefetch(v, op, nxt * TP, min(TP, plim - nxt * TP), RS, RSP, TP, An, An + TP * RSP,
                        scs + (st ^ 1) * 2 * TP, tts + (st ^ 1) * 2 * TP);
        }
        cp_commit();
        cp_wait<1>();
        if (p0 >= v.kpad) {
            if (RS % 4 == 0) {
                __syncthreads();  // the rows' floats, copied by other threads, in shared memory
                ns_widen_rows(op, np, RS, RSP, A, B);
            } else {
                ns_widen(op, np, RS, RSP, A, B);
            }
        }
        __syncthreads();  // this tile's stage (and P) in shared memory
        double val[Q][F];
        if (worker) {
            ns_task<S, !GARLI_SCALE>(op, PL + r * SS, PR + r * SS, A + r * S, B + r * S, RSP, tt, TP, pl, fr, val);
#pragma unroll
            for (int j = 0; j < Q; j++) {
                double m = val[j][0];
#pragma unroll
                for (int k = 1; k < F; k++)
                    if (fg + NF * k < S) m = val[j][k] > m ? val[j][k] : m;
#pragma unroll
                for (int d = 1; d < NF; d <<= 1) {
                    const double o = __shfl_xor_sync(0xffffffffu, m, d);
                    m = o > m ? o : m;
                }
                if (fg == 0) mxr[r * TP + pl[j]] = m;
            }
        }
        __syncthreads();
        // per-pattern largest entry over all rates and states (RescaleRateHetNState, tree.cpp:3492-3598)
        for (int q = threadIdx.x; q < np; q += blockDim.x) {
            double large = mxr[q];
            for (int rr = 1; rr < R; rr++) large = mxr[rr * TP + q] > large ? mxr[rr * TP + q] : large;
            int m = 0;
            if (op.kind == kIntInt) m = sc[q] + sc[TP + q];
            else if (op.kind == kIntTip) m = sc[q];
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
            mx[q] = mult;
            v.scalers[(long long)op.dest * v.npat_pad + p0 + q] = m;
        }
        __syncthreads();
        if (worker) {
#pragma unroll
            for (int j = 0; j < Q; j++) {
                if (pl[j] >= np) continue;
                const double mult = mx[pl[j]];
                if (p0 < v.kpad) {
                    double *dst = cla_ptr<double>(v, op.dest, p0 + pl[j], RS) + r * S;
#pragma unroll
                    for (int k = 0; k < F; k++)
                        if (fg + NF * k < S) dst[fg + NF * k] = mult != 1.0 ? mul(val[j][k], mult) : val[j][k];
                } else {
                    float *dst = cla_ptr<float>(v, op.dest, p0 + pl[j], RS) + r * S;
#pragma unroll
                    for (int k = 0; k < F; k++)
                        if (fg + NF * k < S) {
                            // keyed on the value's offset in the CLA pool: the same rounding in every run
                            const unsigned int key =
                                (unsigned int)((reinterpret_cast<const char *>(dst + fg + NF * k) - v.partials) >> 2);
                            dst[fg + NF * k] = round_stochastic(mult != 1.0 ? mul(val[j][k], mult) : val[j][k], key);
                        }
                }
            }
        }
    }
    cp_wait<0>();
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
    // P, dP, d2P transposed, [matrix][rate][to][from]: the threads of a warp
    // take consecutive "from" states, so each "to" step reads consecutive words
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
