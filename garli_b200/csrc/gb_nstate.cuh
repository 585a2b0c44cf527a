// gb_nstate.cuh -- 20-state (amino acid) and 61-state (codon) kernels.
//
// CUDA-core FP64 versions that keep GARLI's per-site arithmetic order
// (sequential sums over "to" states, tree.cpp:7843-7910, :8537-8600,
// :5597-6460, optimization.cpp:2592-3614).  CLA updates: a block stages the
// op's two P(t) sets in shared memory once and walks pattern tiles, the next
// tile's inputs arriving by cp.async while a register tile per lane (several
// patterns x several from-states) is computed.  Edge evaluations: the same
// structure with the edge's P, dP, d2P; each rate's sum over "from" runs in
// the reference's order through warp shuffles.
#pragma once
#include "gb_common.cuh"
#include "gb_dna.cuh"
#include "gb_stage.cuh"

namespace gb {

// Register tile of the n-state CLA kernel: the 32 lanes of a warp are NF
// "from"-state groups x NQ pattern groups; a lane computes F from-states
// (fg, fg + NF, ...) of Q patterns (qg, qg + NQ, ...) of one rate category, so
// each P entry read from shared memory serves Q patterns and each child value
// serves F from-states.
template <int S, int QP = 2>
struct NsTile {
    static constexpr int NF = S <= 20 ? 4 : 8;
    static constexpr int F = (S + NF - 1) / NF;
    static constexpr int NQ = 32 / NF;
    static constexpr int Q = QP;
    static constexpr int PW = NQ * Q;  // patterns of one warp task; tiles are multiples of it
};
// the edge kernel's tile (two patterns per lane measured faster than one
// with two blocks per SM)
constexpr int kEdgeQ = 2;

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

// Asynchronous copy of n doubles (a block's matrices) into shared memory:
// 16-byte pieces when both addresses are 16-byte aligned and n is even.
__device__ __forceinline__ void stage_doubles(double *dst, const double *src, int n) {
    if (((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15u) == 0 && n % 2 == 0) {
        for (int i = threadIdx.x; i < n / 2; i += blockDim.x) cp16(smem_u32(dst + 2 * i), src + 2 * i);
    } else {
        for (int i = threadIdx.x; i < n; i += blockDim.x) cp8(smem_u32(dst + i), src + i);
    }
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
    stage_doubles(PL, v.mats + (long long)op.p1 * v.mat_stride, RSS);
    stage_doubles(PR, v.mats + (long long)op.p2 * v.mat_stride, RSS);
    cp_commit();
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

// dynamic shared memory of k_edge_ns in bytes: P (and dP, d2P) of the edge,
// two stages of the parent's and the child's tiles, per-(sum, rate, pattern)
// from-sums, frequencies and category probabilities, then per stage the
// scalers, counts and constant states ([stage][4][TP] ints) and the child's
// tip codes ([stage][2][TP] bytes, child in the second half)
__host__ __device__ inline size_t ns_edge_smem_bytes(int S, int R, int TP, bool deriv) {
    const size_t RS = (size_t)R * S, RSP = (size_t)ns_row_stride(R * S);
    const size_t dbl = (deriv ? 3 : 1) * RS * S + 4 * (size_t)TP * RSP + 3 * (size_t)R * TP + S + R;
    return (dbl * 8 + 15) / 16 * 16 + 2 * 4 * (size_t)TP * 4 + 2 * 2 * (size_t)TP;
}

// Edge evaluation for S states (the n-state forms of Tree::GetScore /
// ConditionalLikelihoodRateHet, tree.cpp:5597-6460, and of the derivative
// sums, optimization.cpp:2592-3614): per (pattern, rate, from) the child's
// transition sum l = sum_to P[from][to] * child[to] (dP, d2P for the
// derivatives; a tip child's entry directly), the term
// l * partial[from] * freqs[from], summed over "from" in order per rate, then
// over rates with the category probabilities, plus pinv, log and the
// derivative ratios; per-block sums of count-weighted site values.  The
// per-site arithmetic and order are GARLI's (plain form: separate products
// and sums; precision form: fused multiply-add in the transition sums).
// Structure as k_cla_ns: matrices staged once per block, pattern tiles walked
// grid-stride and double-buffered by cp.async, one warp task (rate, PW
// patterns) per warp with a register tile of F from-states x Q patterns; a
// rate's "from" sum runs in order through warp shuffles.
template <bool GARLI_SCALE, bool DERIV, int S>
__global__ void __launch_bounds__(kThreads, 1) k_edge_ns(View v, int pbuf, int cbuf, int mat, int child_tip,
                                                         int write_sites, int R, int TP) {
    using T = NsTile<S, kEdgeQ>;
    constexpr int NF = T::NF, F = T::F, NQ = T::NQ, Q = T::Q, SS = S * S, NM = DERIV ? 3 : 1;
    extern __shared__ __align__(16) double sm[];
    const int RS = R * S, RSS = R * SS, RSP = ns_row_stride(RS);
    double *M = sm, *stg = M + NM * RSS, *rsum = stg + 4 * TP * RSP, *Fq = rsum + 3 * R * TP, *RP = Fq + S;
    char *tail = reinterpret_cast<char *>(sm) +
                 ((size_t)(NM * RSS + 4 * TP * RSP + 3 * R * TP + S + R) * 8 + 15) / 16 * 16;
    int *scs = reinterpret_cast<int *>(tail);                  // [stage][parent, child, count, const][TP]
    uint8_t *tts = reinterpret_cast<uint8_t *>(scs + 8 * TP);  // [stage][-, child][TP]
    DevOp op;  // the parent as child 1 and the child as child 2 of a CLA op, for the staging helpers
    op.c1 = pbuf;
    op.c2 = cbuf;
    op.kind = child_tip ? kIntTip : kIntInt;
    const int ntiles = (v.npat + TP - 1) / TP;
    auto prefetch = [&](int tile, int st) {
        const int p0 = tile * TP, np = min(TP, v.npat - p0);
        double *A = stg + st * 2 * TP * RSP;
        int *sc = scs + st * 4 * TP;
        ns_prefetch(v, op, p0, np, RS, RSP, TP, A, A + TP * RSP, sc, tts + st * 2 * TP);
        for (int q = threadIdx.x; q < np; q += blockDim.x) {
            cp4(smem_u32(sc + 2 * TP + q), v.counts + p0 + q);
            cp4(smem_u32(sc + 3 * TP + q), v.const_states + p0 + q);
        }
    };
    double accL = 0.0, acc1 = 0.0, acc2 = 0.0;
    if ((int)blockIdx.x < ntiles) {
        prefetch(blockIdx.x, 0);
        stage_doubles(M, v.mats + (long long)mat * v.mat_stride, NM * RSS);
        cp_commit();
        for (int i = threadIdx.x; i < S; i += blockDim.x) Fq[i] = v.freqs[i];
        for (int i = threadIdx.x; i < R; i += blockDim.x) RP[i] = v.rate_probs[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int fg = lane % NF, qg = lane / NF;
    const int tasks = R * (TP / T::PW);  // <= warps of the block (host-chosen TP)
    const bool worker = warp < tasks;
    const int r = worker ? warp % R : 0, pb = worker ? (warp / R) * T::PW : 0;
    int fr[F], pl[Q];
#pragma unroll
    for (int k = 0; k < F; k++) fr[k] = min(fg + NF * k, S - 1);
#pragma unroll
    for (int j = 0; j < Q; j++) pl[j] = pb + qg + NQ * j;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int st = it & 1;
        const int p0 = tile * TP, np = min(TP, v.npat - p0);
        double *A = stg + st * 2 * TP * RSP, *B = A + TP * RSP;  // parent partial, child
        const int *sc = scs + st * 4 * TP;
        const uint8_t *tt = tts + st * 2 * TP;
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) prefetch(nxt, st ^ 1);
        cp_commit();
        cp_wait<1>();
        if (p0 >= v.kpad) {
            if (RS % 4 == 0) {
                __syncthreads();
                ns_widen_rows(op, np, RS, RSP, A, B);
            } else {
                ns_widen(op, np, RS, RSP, A, B);
            }
        }
        __syncthreads();  // this tile's stage (and the matrices) in shared memory
        if (worker) {
            const double *m0 = M + r * SS;
            double tl[Q][F], t1[Q][F], t2[Q][F];
            if (!child_tip) {
                double l[Q][F], a[Q][F], b[Q][F];
#pragma unroll
                for (int j = 0; j < Q; j++)
#pragma unroll
                    for (int k = 0; k < F; k++) l[j][k] = a[j][k] = b[j][k] = 0.0;
                const double *Br = B + r * S;
                if constexpr (S % 2 == 0) {
#pragma unroll 1
                    for (int to = 0; to < S; to += 2) {
                        double2 c[Q];
#pragma unroll
                        for (int j = 0; j < Q; j++) c[j] = *reinterpret_cast<const double2 *>(Br + pl[j] * RSP + to);
#pragma unroll
                        for (int k = 0; k < F; k++) {
                            const double2 p = *reinterpret_cast<const double2 *>(m0 + fr[k] * S + to);
#pragma unroll
                            for (int j = 0; j < Q; j++) {
                                l[j][k] = mac<!GARLI_SCALE>(l[j][k], p.x, c[j].x);
                                l[j][k] = mac<!GARLI_SCALE>(l[j][k], p.y, c[j].y);
                            }
                            if (DERIV) {
                                const double2 p1 = *reinterpret_cast<const double2 *>(m0 + RSS + fr[k] * S + to);
                                const double2 p2 = *reinterpret_cast<const double2 *>(m0 + 2 * RSS + fr[k] * S + to);
#pragma unroll
                                for (int j = 0; j < Q; j++) {
                                    a[j][k] = mac<!GARLI_SCALE>(a[j][k], p1.x, c[j].x);
                                    a[j][k] = mac<!GARLI_SCALE>(a[j][k], p1.y, c[j].y);
                                    b[j][k] = mac<!GARLI_SCALE>(b[j][k], p2.x, c[j].x);
                                    b[j][k] = mac<!GARLI_SCALE>(b[j][k], p2.y, c[j].y);
                                }
                            }
                        }
                    }
                } else {
#pragma unroll 1
                    for (int to = 0; to < S; to++) {
                        double c[Q];
#pragma unroll
                        for (int j = 0; j < Q; j++) c[j] = Br[pl[j] * RSP + to];
#pragma unroll
                        for (int k = 0; k < F; k++) {
                            const double p = m0[fr[k] * S + to];
#pragma unroll
                            for (int j = 0; j < Q; j++) l[j][k] = mac<!GARLI_SCALE>(l[j][k], p, c[j]);
                            if (DERIV) {
                                const double p1 = m0[RSS + fr[k] * S + to], p2 = m0[2 * RSS + fr[k] * S + to];
#pragma unroll
                                for (int j = 0; j < Q; j++) {
                                    a[j][k] = mac<!GARLI_SCALE>(a[j][k], p1, c[j]);
                                    b[j][k] = mac<!GARLI_SCALE>(b[j][k], p2, c[j]);
                                }
                            }
                        }
                    }
                }
                // reference: temp * partial[from] * freqs[from]
#pragma unroll
                for (int j = 0; j < Q; j++)
#pragma unroll
                    for (int k = 0; k < F; k++) {
                        const double w = A[pl[j] * RSP + r * S + fr[k]], f = Fq[fr[k]];
                        tl[j][k] = mul(mul(l[j][k], w), f);
                        t1[j][k] = DERIV ? mul(mul(a[j][k], w), f) : 0.0;
                        t2[j][k] = DERIV ? mul(mul(b[j][k], w), f) : 0.0;
                    }
            } else {
#pragma unroll
                for (int j = 0; j < Q; j++) {
                    const int s = tt[TP + pl[j]];
#pragma unroll
                    for (int k = 0; k < F; k++) {
                        const double w = A[pl[j] * RSP + r * S + fr[k]], f = Fq[fr[k]];
                        if (s < S) {
                            tl[j][k] = mul(mul(m0[fr[k] * S + s], w), f);
                            t1[j][k] = DERIV ? mul(mul(m0[RSS + fr[k] * S + s], w), f) : 0.0;
                            t2[j][k] = DERIV ? mul(mul(m0[2 * RSS + fr[k] * S + s], w), f) : 0.0;
                        } else {
                            // total ambiguity: partial[from] * freqs[from], no derivative terms
                            tl[j][k] = mul(w, f);
                            t1[j][k] = DERIV ? mul(mul(0.0, w), f) : 0.0;
                            t2[j][k] = DERIV ? mul(mul(0.0, w), f) : 0.0;
                        }
                    }
                }
            }
            // this rate's sums over "from", in order: the value of "from" lives in
            // lane (qg, from % NF), register from / NF
#pragma unroll
            for (int j = 0; j < Q; j++) {
                double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
                for (int from = 0; from < S; from++) {
                    const int src = qg * NF + from % NF;
                    s0 = add(s0, __shfl_sync(0xffffffffu, tl[j][from / NF], src));
                    if (DERIV) {
                        s1 = add(s1, __shfl_sync(0xffffffffu, t1[j][from / NF], src));
                        s2 = add(s2, __shfl_sync(0xffffffffu, t2[j][from / NF], src));
                    }
                }
                if (fg == 0) {
                    rsum[r * TP + pl[j]] = s0;
                    rsum[(R + r) * TP + pl[j]] = s1;
                    rsum[(2 * R + r) * TP + pl[j]] = s2;
                }
            }
        }
        __syncthreads();
        for (int q = threadIdx.x; q < np; q += blockDim.x) {
            const int p = p0 + q;
            double siteL = 0.0, sD1 = 0.0, sD2 = 0.0;
            for (int rr = 0; rr < R; rr++) {
                siteL = add(siteL, mul(rsum[rr * TP + q], RP[rr]));
                if (DERIV) {
                    sD1 = add(sD1, mul(rsum[(R + rr) * TP + q], RP[rr]));
                    sD2 = add(sD2, mul(rsum[(2 * R + rr) * TP + q], RP[rr]));
                }
            }
            const int m1 = sc[q];
            const int m2 = child_tip ? 0 : sc[TP + q];
            const int cs = sc[3 * TP + q];
            if (v.has_pinv && cs >= 0) {
                const double pf = mul(v.pinv, Fq[cs]);
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
                const double cnt = (double)sc[2 * TP + q];
                accL = add(accL, mul(u, cnt));
                if (DERIV) {
                    acc1 = add(acc1, mul(cnt, d1));
                    acc2 = add(acc2, mul(cnt, d2));
                }
            }
        }
        __syncthreads();  // the stage's scalers read before the next prefetch overwrites them
    }
    cp_wait<0>();
    block_sum3(accL, acc1, acc2, v.block_sums + 3 * blockIdx.x);
}

}  // namespace gb
