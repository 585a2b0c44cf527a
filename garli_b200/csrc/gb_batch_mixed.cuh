// gb_batch_mixed.cuh -- the precision form's batched candidate pass.
//
// The command queue of k_batch4 (gb_batch.cuh), laid out for throughput and
// run as one CUDA graph of three kernels:
//   k_level4m (kBLevel, one launch per level): CLA updates with one lane per
//             (pattern, category), the op's P blocks in padded shared memory,
//             FP64 fused arithmetic, the pattern's power-of-two
//             normalisation by a shuffle max, FP32 stores with an 8-bit
//             mantissa extension (unbiased stochastic rounding of the
//             extension byte, exact, no division); every lane prefetches its
//             inputs two tiles ahead with cp.async.
//   k_coef4m  (kBCoef, one launch per step): for every candidate's step, the
//             spectral coefficients of the branch it optimises.  With
//             P_r(t) = U diag(exp(s_rk t)) U^-1, s_rk = lambda_k rate_r / (1 - pinv),
//               L_p(t) = sum_rk A[p,r,k] exp(s_rk t) (+ the +I term), with
//               A[p,r,k] = w_r (sum_i pi_i W[p,r,i] U[i,k]) (sum_j U^-1[k,j] V[p,r,j]),
//             where W = (P_o1 V_o1) o (P_o2 V_o2) is the partial on the
//             connector's side, formed in FP64 registers and never stored,
//             and V the CLA (or tip) across the branch.  One lane per
//             (pattern, category).  A is FP64.  A reversible rate matrix's
//             rows sum to zero, so one eigenvalue lambda_k0 is zero (to
//             rounding) and exp(s_rk0 t) = 1 for every category and length:
//             its R coefficients are stored as one sum, 1 + 3R per pattern,
//             laid out [slot][q][pattern] with q = 0 the stationary sum and
//             q = 1 + 3r + j the j-th other eigenvalue of category r; the
//             site's scale exponent is m_o1 + m_o2 + m_V.
//   k_batch4m (the kBNewton / kBScore runs between them, persistent):
//             Newton-Raphson in lockstep; an iteration reads only A:
//             L = A_0 + sum A e, dL/dt = sum A s e, d2L/dt2 = sum A s^2 e with the
//             per-candidate tables e, s e, s^2 e recomputed in FP64 after
//             every step.  A chunk = 256 patterns summed by one warp (8 per
//             lane, then a shuffle tree) -- no block barrier; the candidate's
//             chunk sums are reduced by one warp in a fixed order.  kBScore:
//             the same sweep at the optimised lengths.
// The level and coefficient kernels fit 64 registers a thread (4 CTAs per
// SM); the persistent kernel's sweeps need 120 (2 CTAs per SM).
// lnL, d1, d2 accumulate in FP64; the Newton step and P(t) are FP64.
#pragma once
#include "gb_batch.cuh"
#include "gb_stage.cuh"

namespace gb {

enum : int { kBCoef = 4 };

// a step in the precision form: the two other sides (buffer or tip, matrix;
// m2 < 0: side 1 is the partial itself, no matrix) and the side across the branch
struct MEntry {
    int b1, t1, m1;
    int b2, t2, m2;
    int bk, tk, mk;
    int wide;  // FP64 (wide) buffers: bit 0 side 1, bit 1 side 2, bit 2 the side across the branch
};

struct MixedArgs {
    const BCmd *cmds;
    int ncmd;
    const DevOp *ops;
    const MEntry *entries;
    BSlot *slots;
    NrParams prm;
    double *lengths;
    const double *eig;    // lambda (scaled), U, U^-1
    const double *rates;
    double *coef;         // [slot][1 + 3R][npat_pad]
    int *cscale;          // max_entries x npat_pad
    double *etab;         // max_entries x 3 x (1 + 3R)
    double *chunk_sums;   // max_entries x nchunks x 3
    int *active;
    int *nactive;
    int max_entries;
    GridSync *gs;
    int tiles_per_item;   // CLA / coefficient work item: this many tiles of 256/G patterns
    int chunks_per_item;  // sweep work item: this many 256-pattern chunks per warp
    unsigned long long *trace;
    int trace_cap;
};

// Power-of-two normalisation of one pattern-category slice d[4] (the max over
// the pattern's G lanes) and its store: FP64 segment as is, FP32 segment as
// FP32 + extension byte (ext_encode4).  All G lanes of the pattern must call
// this together.
template <int R>
__device__ __forceinline__ void cla_finish_m(const View &v, int dest, bool wide, int p, int r, bool act, double d[4],
                                             int m) {
    constexpr int G = Lanes<R>::G;
    double mx = act ? fmax(fmax(d[0], d[1]), fmax(d[2], d[3])) : 0.0;
#pragma unroll
    for (int o = 1; o < G; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (!act) return;
    int e = 0;
    if (mx > 0.0) e = max(-1000, min(1000, ilogb(mx)));
    const double sc = pow2d(-e);
#pragma unroll
    for (int k = 0; k < 4; k++) d[k] *= sc;
    if (wide) {
        st4d(cla_ptr_wide(v, dest, p, R * 4) + r * 4, d);
    } else if (p < v.kpad) {
        st4d(cla_ptr<double>(v, dest, p, R * 4) + r * 4, d);
    } else {
        float *q = cla_ptr<float>(v, dest, p, R * 4) + r * 4;
        // keyed on the slice's offset in the CLA pool: the same rounding in every run
        const unsigned int key = (unsigned int)((reinterpret_cast<const char *>(q) - v.partials) >> 4);
        float4 hi;
        unsigned int e;
        ext_encode4(d, key, hi, e);
        reinterpret_cast<float4 *>(q)[0] = hi;
        cla_ext(v, dest, p, R * 4)[r] = e;
    }
    if (r == 0) v.scalers[(long long)dest * v.npat_pad + p] = m - e;
}

// (P c) for the 4 states of one category (P: that category's 4x4 block,
// 16-byte aligned, read as pairs), FP64 fused
__device__ __forceinline__ void pvec(const double *P, const double c[4], double out[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const double2 lo = *reinterpret_cast<const double2 *>(P + i * 4);
        const double2 hi = *reinterpret_cast<const double2 *>(P + i * 4 + 2);
        out[i] = fma(hi.y, c[3], fma(hi.x, c[2], fma(lo.y, c[1], lo.x * c[0])));
    }
}
__device__ __forceinline__ void pvec_tip(const double *P, int code, double out[4]) {
    code &= 15;
    if ((code & (code - 1)) == 0 && code) {
        // one state: a column of P (the sum below with its zero terms dropped)
        const int b = __ffs(code) - 1;
#pragma unroll
        for (int i = 0; i < 4; i++) out[i] = P[i * 4 + b];
        return;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < 4; b++)
            if (code & (1 << b)) s += P[i * 4 + b];
        out[i] = (code == 15 || code == 0) ? 1.0 : s;
    }
}

// Child slice of category r at pattern p in FP64: a wide (FP64) buffer or
// the FP64 segment holds doubles, the FP32 segment floats and their extension bytes.
template <int R>
__device__ __forceinline__ void slice_load(const View &v, int b, bool wide, int p, int r, double c[4]) {
    if (wide) {
        ld4d_cg(cla_ptr_wide(v, b, p, R * 4) + r * 4, c);
    } else if (p < v.kpad) {
        ld4d_cg(cla_ptr<double>(v, b, p, R * 4) + r * 4, c);
    } else {
        const float4 a = __ldcg(reinterpret_cast<const float4 *>(cla_ptr<float>(v, b, p, R * 4) + r * 4));
        ext_decode4(a, __ldcg(cla_ext(v, b, p, R * 4) + r), c);
    }
}

// CLA update of tiles [t0, t1) of one op; lane = category r of pattern
// tile * PPB + threadIdx.x / G; PL, PR = the category's P blocks in shared
// memory.  Both children's loads of a tile are issued before its arithmetic;
// one tile at a time: holding a second tile's loads in flight spilled
// registers in the batched kernel and measured slower.
template <int R>
__device__ __forceinline__ void cla_tiles_m(const View &v, const DevOp &op, const double *PL, const double *PR,
                                            int t0, int t1, int r, bool lane_ok) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    const int pl = threadIdx.x / G;
    const bool w1 = op.wide & kWideC1, w2 = op.wide & kWideC2, wd = op.wide & kWideDest;
    for (int tile = t0; tile < t1; tile++) {
        const int p = tile * PPB + pl;
        const bool act = lane_ok && p < v.npat;
        double a[4], b[4], d[4] = {0, 0, 0, 0};
        int m = 0;
        unsigned char c1 = 15, c2 = 15;
        if (act) {
            if (op.kind == kTipTip) {
                c1 = v.tips[(long long)op.c1 * v.npat_pad + p];
                c2 = v.tips[(long long)op.c2 * v.npat_pad + p];
            } else {
                slice_load<R>(v, op.c1, w1, p, r, a);
                m = __ldcg(v.scalers + (long long)op.c1 * v.npat_pad + p);
                if (op.kind == kIntInt) {
                    slice_load<R>(v, op.c2, w2, p, r, b);
                    m += __ldcg(v.scalers + (long long)op.c2 * v.npat_pad + p);
                } else {
                    c2 = v.tips[(long long)op.c2 * v.npat_pad + p];
                }
            }
            double x[4], y[4];
            if (op.kind == kTipTip) pvec_tip(PL, c1, x);
            else pvec(PL, a, x);
            if (op.kind == kIntInt) pvec(PR, b, y);
            else pvec_tip(PR, c2, y);
#pragma unroll
            for (int k = 0; k < 4; k++) d[k] = x[k] * y[k];
        }
        cla_finish_m<R>(v, op.dest, wd, p, r, act, d, m);
    }
}

// ---------------------------------------------------------------------------
// Prefetched CLA tiles: every lane copies its own inputs of the tiles ahead
// into its own shared-memory slots with asynchronous copies (cp.async, 16
// bytes, through L2), kCpStages - 1 tiles ahead of the arithmetic, so a lane
// keeps the next tile's loads in flight without holding them in registers and
// without block barriers (a lane reads only what it copied).  Two stages at 4
// CTAs per SM measured faster than three at 3.  Per lane and
// stage: child 1's slice (32 B), child 2's slice (32 B), and two 16-byte
// words holding the pattern's scale exponents (the aligned 16-byte block that
// contains it).  Tip codes are not copied.  Layout [stage][field][lane].
constexpr int kCpStages = 2;
constexpr int kCpLane = 96;  // bytes per lane and stage
__host__ __device__ constexpr int cp_smem_bytes() { return kCpStages * kCpLane * kThreads; }

struct CpSlots {
    unsigned char *a, *b, *c, *d;  // this lane's slots of one stage
};
__device__ __forceinline__ CpSlots cp_slots(unsigned char *cps, int stage) {
    unsigned char *s = cps + stage * kCpLane * kThreads;
    const int t = threadIdx.x;
    return {s + t * 32, s + 32 * kThreads + t * 32, s + 64 * kThreads + t * 16, s + 80 * kThreads + t * 16};
}

// the copies of tile `tile` for this lane (none past t1 or for an idle lane), one commit group
template <int R>
__device__ __forceinline__ void cp_issue(const View &v, const DevOp &op, int tile, int t1, int r, bool lane_ok,
                                         unsigned char *cps, int stage) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    const int p = tile * PPB + threadIdx.x / G;
    if (lane_ok && tile < t1 && p < v.npat) {
        const CpSlots sl = cp_slots(cps, stage);
        auto slice = [&](unsigned char *dst, int b, bool wide) {
            if (wide || p < v.kpad) {
                const double *src = (wide ? cla_ptr_wide(v, b, p, R * 4) : cla_ptr<double>(v, b, p, R * 4)) + r * 4;
                cp16(smem_u32(dst), src);
                cp16(smem_u32(dst + 16), src + 2);
            } else {
                cp16(smem_u32(dst), cla_ptr<float>(v, b, p, R * 4) + r * 4);
                cp4(smem_u32(dst + 16), cla_ext(v, b, p, R * 4) + r);
            }
        };
        // tip codes are read directly at the arithmetic (one byte, shared by the
        // pattern's lanes and its neighbours: a copy per lane would repeat it)
        if (op.kind != kTipTip) {
            // the scale exponents only for the lane of category 0 (the one that stores the sum)
            slice(sl.a, op.c1, op.wide & kWideC1);
            if (r == 0) cp16(smem_u32(sl.c), v.scalers + (long long)op.c1 * v.npat_pad + (p & ~3));
            if (op.kind == kIntInt) {
                slice(sl.b, op.c2, op.wide & kWideC2);
                if (r == 0) cp16(smem_u32(sl.d), v.scalers + (long long)op.c2 * v.npat_pad + (p & ~3));
            }
        }
    }
    cp_commit();
}

// CLA update of tiles [t0, t1) of one op from prefetched inputs; the
// arithmetic of cla_tiles_m
template <int R>
__device__ __forceinline__ void cla_tiles_cp(const View &v, const DevOp &op, const double *PL, const double *PR,
                                             int t0, int t1, int r, bool lane_ok, unsigned char *cps) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    const int pl = threadIdx.x / G;
#pragma unroll
    for (int q = 0; q < kCpStages - 1; q++) cp_issue<R>(v, op, t0 + q, t1, r, lane_ok, cps, q);
    int stage = 0;
    for (int tile = t0; tile < t1; tile++) {
        cp_issue<R>(v, op, tile + kCpStages - 1, t1, r, lane_ok, cps, stage == 0 ? kCpStages - 1 : stage - 1);
        cp_wait<kCpStages - 1>();
        const int p = tile * PPB + pl;
        const bool act = lane_ok && p < v.npat;
        double d[4] = {0, 0, 0, 0};
        int m = 0;
        if (act) {
            const CpSlots sl = cp_slots(cps, stage);
            auto slice = [&](const unsigned char *src, bool wide, double out[4]) {
                if (wide || p < v.kpad) {
                    const double2 x = *reinterpret_cast<const double2 *>(src);
                    const double2 y = *reinterpret_cast<const double2 *>(src + 16);
                    out[0] = x.x;
                    out[1] = x.y;
                    out[2] = y.x;
                    out[3] = y.y;
                } else {
                    ext_decode4(*reinterpret_cast<const float4 *>(src),
                                *reinterpret_cast<const unsigned int *>(src + 16), out);
                }
            };
            double a[4], b[4], x[4], y[4];
            if (op.kind == kTipTip) {
                pvec_tip(PL, __ldg(v.tips + (long long)op.c1 * v.npat_pad + p), x);
                pvec_tip(PR, __ldg(v.tips + (long long)op.c2 * v.npat_pad + p), y);
            } else {
                slice(sl.a, op.wide & kWideC1, a);
                if (r == 0) m = reinterpret_cast<const int *>(sl.c)[p & 3];
                pvec(PL, a, x);
                if (op.kind == kIntInt) {
                    slice(sl.b, op.wide & kWideC2, b);
                    if (r == 0) m += reinterpret_cast<const int *>(sl.d)[p & 3];
                    pvec(PR, b, y);
                } else {
                    pvec_tip(PR, __ldg(v.tips + (long long)op.c2 * v.npat_pad + p), y);
                }
            }
#pragma unroll
            for (int k = 0; k < 4; k++) d[k] = x[k] * y[k];
        }
        cla_finish_m<R>(v, op.dest, op.wide & kWideDest, p, r, act, d, m);
        stage = stage == kCpStages - 1 ? 0 : stage + 1;
    }
}

// One side of a coefficient entry for lane category r at pattern p: the child
// slice in FP64 or the tip code, loaded before any arithmetic.
struct SideRaw {
    double c[4];
    int code, scale;
};
template <int R>
__device__ __forceinline__ void side_load(const View &v, int b, int tip, bool wide, int p, int r, SideRaw &s) {
    s.c[0] = s.c[1] = s.c[2] = s.c[3] = 0.0;
    s.code = 15;
    s.scale = 0;
    if (b < 0) return;
    if (tip) {
        s.code = v.tips[(long long)b * v.npat_pad + p];
        return;
    }
    slice_load<R>(v, b, wide, p, r, s.c);
    if (r == 0) s.scale = __ldcg(v.scalers + (long long)b * v.npat_pad + p);  // only category 0 stores it
}
// the side's vector (P_s V_s) (or V_s itself when it has no matrix), FP64
__device__ __forceinline__ void side_vec(const double c[4], int code, int tip, const double *P, double out[4]) {
    if (tip) {
        if (P) {
            pvec_tip(P, code, out);
        } else {
            code &= 15;
#pragma unroll
            for (int k = 0; k < 4; k++) out[k] = (code == 15 || code == 0 || (code >> k) & 1) ? 1.0 : 0.0;
        }
    } else if (P) {
        pvec(P, c, out);
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) out[k] = c[k];
    }
}

// coefficients per pattern: the stationary sum and 3 per category
template <int R>
struct Coefs {
    static constexpr int N = 1 + 3 * R;
};

// the stationary eigenvalue: the one of least magnitude
__device__ __forceinline__ int stationary_index(const double *eig) {
    int k0 = 0;
    double m = fabs(__ldg(eig));
#pragma unroll
    for (int k = 1; k < 4; k++) {
        const double a = fabs(__ldg(eig + k));
        if (a < m) {
            m = a;
            k0 = k;
        }
    }
    return k0;
}

// Coefficients of category r at pattern p from the three side vectors, stored
// to the entry's slot: the 3 non-stationary ones of the lane's category, and
// the stationary one summed over the pattern's G lanes (lane_ok false: a
// zero share).  All G lanes of the pattern must call this together.
template <int R>
__device__ __forceinline__ void coef_store(const View &v, const MixedArgs &A, int slot, int p, int r, bool act,
                                           const double x[4], const double y[4], const double z[4], int scale,
                                           const double *sU, const double *sUi, int k0) {
    constexpr int G = Lanes<R>::G;
    constexpr int NC = Coefs<R>::N;
    double w[4], c[4];
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = x[i] * y[i] * v.freqs[i];
    const double rp = act ? v.rate_probs[r] : 0.0;
    // U and U^-1 (16-byte aligned, row-major) read as pairs
    double U[16], Ui[16];
#pragma unroll
    for (int q = 0; q < 8; q++) {
        const double2 u = reinterpret_cast<const double2 *>(sU)[q];
        const double2 ui = reinterpret_cast<const double2 *>(sUi)[q];
        U[2 * q] = u.x;
        U[2 * q + 1] = u.y;
        Ui[2 * q] = ui.x;
        Ui[2 * q + 1] = ui.y;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double a_k = fma(w[3], U[12 + k], fma(w[2], U[8 + k], fma(w[1], U[4 + k], w[0] * U[k])));
        const double b_k = fma(Ui[k * 4 + 3], z[3], fma(Ui[k * 4 + 2], z[2], fma(Ui[k * 4 + 1], z[1], Ui[k * 4] * z[0])));
        c[k] = act ? rp * a_k * b_k : 0.0;
    }
    double c0 = c[0];
#pragma unroll
    for (int k = 1; k < 4; k++)
        if (k == k0) c0 = c[k];
#pragma unroll
    for (int o = 1; o < G; o <<= 1) c0 += __shfl_xor_sync(0xffffffffu, c0, o);
    if (!act) return;
    double *out = A.coef + (long long)slot * NC * v.npat_pad + p;
    int j = 0;
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (k != k0) out[(long long)(1 + 3 * r + j++) * v.npat_pad] = c[k];
    if (r == 0) {
        out[0] = c0;
        A.cscale[(long long)slot * v.npat_pad + p] = scale;
    }
}

// Coefficient pass of tiles [t0, t1) of one entry; lane = category r of
// pattern tile * PPB + threadIdx.x / G.  P1, P2 = the sides' P blocks of
// category r (null: no matrix), sU / sUi = U and U^-1 in shared memory.  One
// tile per load batch: three sides' slices per lane already fill the registers.
template <int R>
__device__ __forceinline__ void coef_tiles_m(const View &v, const MixedArgs &A, const MEntry &en, const double *P1,
                                             const double *P2, const double *sU, const double *sUi, int slot, int t0,
                                             int t1, int r, bool lane_ok, int k0) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    const int pl = threadIdx.x / G;
    const bool w1 = en.wide & 1, w2 = en.wide & 2, wk = en.wide & 4;
    for (int tile = t0; tile < t1; tile++) {
        const int p = tile * PPB + pl;
        const bool act = lane_ok && p < v.npat;
        SideRaw S1, S2, SK;
        side_load<R>(v, act ? en.b1 : -1, en.t1, w1, p, r, S1);
        side_load<R>(v, act ? en.b2 : -1, en.t2, w2, p, r, S2);
        side_load<R>(v, act ? en.bk : -1, en.tk, wk, p, r, SK);
        double x[4] = {0, 0, 0, 0}, y[4] = {1, 1, 1, 1}, z[4] = {0, 0, 0, 0};
        if (act) {
            side_vec(S1.c, S1.code, en.t1, P1, x);
            if (en.b2 >= 0) side_vec(S2.c, S2.code, en.t2, P2, y);
            side_vec(SK.c, SK.code, en.tk, nullptr, z);
        }
        coef_store<R>(v, A, slot, p, r, act, x, y, z, S1.scale + S2.scale + SK.scale, sU, sUi, k0);
    }
}

// e, s e, s^2 e of every stored coefficient at length t, by one warp, into
// etab[3][1 + 3R]; the stationary one is exactly (1, 0, 0)
template <int R>
__device__ __forceinline__ void etab_warp(const double *eig, const double *rates, double pinv, int has_pinv, double t,
                                          double *etab) {
    constexpr int NC = Coefs<R>::N;
    const int lane = threadIdx.x & 31;
    const int k0 = stationary_index(eig);
    for (int q = lane; q < NC; q += 32) {
        double e = 1.0, se = 0.0, s2e = 0.0;
        if (q > 0) {
            const int r = (q - 1) / 3, j = (q - 1) % 3;
            const int k = j < k0 ? j : j + 1;
            double s = __ldcg(eig + k) * __ldcg(rates + r);
            if (has_pinv) s = s / (1.0 - pinv);
            e = exp(s * t);
            se = s * e;
            s2e = s * se;
        }
        etab[q] = e;
        etab[NC + q] = se;
        etab[2 * NC + q] = s2e;
    }
}

// One warp sums a 256-pattern chunk of one entry: lnL, d1, d2 into sums[0..2].
template <int R>
__device__ __forceinline__ void sweep_chunk(const View &v, const MixedArgs &A, int slot, const double *E, int c,
                                            double *sums) {
    const int lane = threadIdx.x & 31;
    constexpr int NC = Coefs<R>::N;
    double aL = 0.0, a1 = 0.0, a2 = 0.0;
    const double *cf = A.coef + (long long)slot * NC * v.npat_pad;
    const int *cs = A.cscale + (long long)slot * v.npat_pad;
#pragma unroll 2
    for (int j = 0; j < 8; j++) {
        const int p = c * 256 + j * 32 + lane;
        if (p >= v.npat) break;
        double L = __ldcg(cf + p), D1 = 0.0, D2 = 0.0;
#pragma unroll
        for (int q = 1; q < NC; q++) {
            const double a = __ldcg(cf + (long long)q * v.npat_pad + p);
            L = fma(a, E[q], L);
            D1 = fma(a, E[NC + q], D1);
            D2 = fma(a, E[2 * NC + q], D2);
        }
        const int m = __ldcg(cs + p);
        const int cb = v.const_states[p];
        if (v.has_pinv && cb >= 0) {
            double btot = 0.0;
#pragma unroll
            for (int s = 0; s < 4; s++)
                if (cb & (1 << s)) btot += v.freqs[s];
            L += ldexp(v.pinv * btot, m);
        }
        const double cnt = (double)v.counts[p];
        const double inv = 1.0 / L;
        const double sd1 = D1 * inv;
        aL = fma(cnt, log(L) - (double)m * 0.69314718055994530941723212145818, aL);
        a1 = fma(cnt, sd1, a1);
        a2 = fma(cnt, fma(D2, inv, -sd1 * sd1), a2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        aL += __shfl_xor_sync(0xffffffffu, aL, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (lane == 0) {
        sums[0] = aL;
        sums[1] = a1;
        sums[2] = a2;
    }
}

// P blocks of the current CLA op: [matrix][category][4x4 + 2 pad] (the pad
// keeps the categories of a warp in different banks for 16-byte reads)
constexpr int kPStride = 18;

// A precision-form CLA level as a launch of its own (the per-tree path and the
// graph-resident pass): the batched kernel's CLA code, blockIdx.y = the op, the
// block's P blocks in shared memory, grid-stride over groups of kCla4mTiles tiles.
constexpr int kCla4mTiles = 4;
template <int R>
__global__ void __launch_bounds__(kThreads, 2) k_cla4m(View v, LevelOps ops) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    __shared__ __align__(16) double sP[2][R][kPStride];
    const DevOp op = ops.op[blockIdx.y];
    for (int q = threadIdx.x; q < 2 * R * 16; q += blockDim.x) {
        const int mi = q / (R * 16), rem = q % (R * 16);
        sP[mi][rem / 16][rem % 16] = __ldcg(v.mats + (long long)(mi ? op.p2 : op.p1) * v.mat_stride + rem);
    }
    __syncthreads();
    const int cr = threadIdx.x % G;
    const bool ok = cr < R;
    const int crr = ok ? cr : 0;
    const int ntiles = (v.npat + PPB - 1) / PPB;
    for (int t0 = blockIdx.x * kCla4mTiles; t0 < ntiles; t0 += gridDim.x * kCla4mTiles)
        cla_tiles_m<R>(v, op, sP[0][crr], sP[1][crr], t0, min(ntiles, t0 + kCla4mTiles), crr, ok);
}

// The CLA levels of a batched pass as launches of their own, one per level
// ahead of the persistent kernel (same stream, same graph): the level code
// alone fits 64 registers, so 4 CTAs share an SM instead of the persistent
// kernel's 2 (its sweeps need 120).  blockIdx.y = the
// op, blockIdx.x = a run of tpi tiles, inputs prefetched as in the persistent
// kernel's levels.
template <int R>
__device__ __forceinline__ void level4m_body(const View &v, const DevOp &op, int tpi) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    __shared__ __align__(16) double sP[2][R][kPStride];
    extern __shared__ __align__(128) unsigned char dsm[];  // cp_smem_bytes() of prefetch slots
    for (int q = threadIdx.x; q < 2 * R * 16; q += blockDim.x) {
        const int mi = q / (R * 16), rem = q % (R * 16);
        sP[mi][rem / 16][rem % 16] = __ldcg(v.mats + (long long)(mi ? op.p2 : op.p1) * v.mat_stride + rem);
    }
    __syncthreads();
    const int cr = threadIdx.x % G;
    const bool ok = cr < R;
    const int crr = ok ? cr : 0;
    const int ctiles = (v.npat + PPB - 1) / PPB;
    const int t0 = blockIdx.x * tpi;
    cla_tiles_cp<R>(v, op, sP[0][crr], sP[1][crr], t0, min(ctiles, t0 + tpi), crr, ok, dsm);
}
template <int R>
__global__ void __launch_bounds__(kThreads, 4) k_level4m(View v, const DevOp *ops, int tpi) {
    level4m_body<R>(v, ops[blockIdx.y], tpi);
}
// the same level launch with the ops passed by value (the per-tree precision
// form: its levels come from gb_update_partials, not a device queue)
template <int R>
__global__ void __launch_bounds__(kThreads, 4) k_level4m_ops(View v, LevelOps ops, int tpi) {
    level4m_body<R>(v, ops.op[blockIdx.y], tpi);
}

// A coefficient pass as a launch of its own, between the persistent kernel's
// Newton commands: blockIdx.y = the entry, blockIdx.x = a run of tpi tiles.
template <int R>
__global__ void __launch_bounds__(kThreads, 4) k_coef4m(View v, MixedArgs A, int first_entry, int tpi) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    __shared__ __align__(16) double sP[2][R][kPStride];
    __shared__ __align__(16) double sUU[32];
    const int e = blockIdx.y;
    const MEntry en = A.entries[first_entry + e];
    for (int q = threadIdx.x; q < 2 * R * 16; q += blockDim.x) {
        const int mi = q / (R * 16), rem = q % (R * 16);
        const int mat = mi ? en.m2 : en.m1;
        sP[mi][rem / 16][rem % 16] = mat >= 0 ? __ldcg(v.mats + (long long)mat * v.mat_stride + rem) : 0.0;
    }
    for (int q = threadIdx.x; q < 32; q += blockDim.x) sUU[q] = __ldg(A.eig + 4 + q);
    __syncthreads();
    const int cr = threadIdx.x % G;
    const bool ok = cr < R;
    const int crr = ok ? cr : 0;
    const int ctiles = (v.npat + PPB - 1) / PPB;
    const int t0 = blockIdx.x * tpi;
    coef_tiles_m<R>(v, A, en, en.m1 >= 0 ? sP[0][crr] : nullptr, en.m2 >= 0 ? sP[1][crr] : nullptr, sUU, sUU + 16, e,
                    t0, min(ctiles, t0 + tpi), crr, ok, stationary_index(A.eig));
}

template <int R>
__global__ void __launch_bounds__(kThreads, 2) k_batch4m(View v, MixedArgs A) {
    constexpr int NC = Coefs<R>::N;
    __shared__ double sE[8][3 * NC];  // one E table per warp
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nchunks = (v.npat + 255) / 256;
    const int gwarp = blockIdx.x * (kThreads / 32) + warp;
    const int nwarps = gridDim.x * (kThreads / 32);
    int ntr = 0;
    auto mark = [&](int code, int na) {
        if (A.trace && blockIdx.x == 0 && threadIdx.x == 0 && ntr < A.trace_cap)
            A.trace[ntr++] = ((unsigned long long)code << 56) | ((unsigned long long)(na & 0xffff) << 40) |
                             (global_ns() & ((1ULL << 40) - 1));
    };
    for (int ci = 0; ci < A.ncmd; ci++) {
        const BCmd cmd = A.cmds[ci];
        mark(kBtNewton, cmd.b);
        const int n = cmd.b;
        const MEntry *ents = A.entries + cmd.a;
        BSlot *slots = A.slots + cmd.a;
        const bool newton = cmd.type == kBNewton;
        // start: Newton states and e tables at the current lengths, everyone active
        for (int e = gwarp; e < n; e += nwarps) {
            const double t = __ldcg(A.lengths + ents[e].mk);
            if (newton && lane == 0) {
                nr_init(slots[e].st, t, A.prm.min_brlen, A.prm.max_brlen);
                slots[e].evals = 0;
            }
            etab_warp<R>(A.eig, A.rates, v.pinv, v.has_pinv, t, A.etab + (long long)e * 3 * NC);
            if (lane == 0) A.active[e] = e;
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
            // (A) sweeps: a warp takes (entry, run of chunks)
            const int cpi = A.chunks_per_item;
            const int items_per_entry = (nchunks + cpi - 1) / cpi;
            const long long nitems = (long long)na * items_per_entry;
            int loaded = -1;
            for (long long item = gwarp; item < nitems; item += nwarps) {
                const int k = (int)(item / items_per_entry);
                const int c0 = (int)(item % items_per_entry) * cpi;
                const int e = __ldcg(act + k);
                if (e != loaded) {
                    loaded = e;
                    __syncwarp();
                    for (int q = lane; q < 3 * NC; q += 32) sE[warp][q] = __ldcg(A.etab + (long long)e * 3 * NC + q);
                    __syncwarp();
                }
                const int c1 = min(nchunks, c0 + cpi);
                for (int c = c0; c < c1; c++)
                    sweep_chunk<R>(v, A, e, sE[warp], c, A.chunk_sums + ((long long)k * nchunks + c) * 3);
            }
            if (!grid_barrier(A.gs, v.status)) return;
            mark(kBtSweepDone, na);
            if (blockIdx.x == 0 && threadIdx.x == 0) A.nactive[cur] = 0;
            // (B) one warp per active entry
            const int nxt = cur ^ 1;
            for (int k = gwarp; k < na; k += nwarps) {
                const int e = __ldcg(act + k);
                double L, d1, d2;
                warp_sum_chunks(A.chunk_sums + (long long)k * nchunks * 3, nchunks, L, d1, d2);
                int fin = 1;
                double t = 0.0;
                if (lane == 0) {
                    BSlot &s = slots[e];
                    if (newton) {
                        if (s.evals == 0) s.first_lnL = L;
                        s.lnL = L;
                        s.d1 = d1;
                        s.d2 = d2;
                        s.evals++;
                        fin = nr_step(s.st, d1, d2, L, A.prm.precision, A.prm.min_brlen, A.prm.max_brlen);
                        A.lengths[ents[e].mk] = s.st.v;
                        t = s.st.v;
                    } else {
                        s.score = L;
                    }
                }
                if (newton) {
                    fin = __shfl_sync(0xffffffffu, fin, 0);
                    t = __shfl_sync(0xffffffffu, t, 0);
                    etab_warp<R>(A.eig, A.rates, v.pinv, v.has_pinv, t, A.etab + (long long)e * 3 * NC);
                    pmat4_warp<R>(A.eig, A.rates, v.pinv, v.has_pinv, t,
                                  const_cast<double *>(v.mats) + (long long)ents[e].mk * v.mat_stride);
                    if (!fin && lane == 0) {
                        const int idx = atomicAdd(A.nactive + nxt, 1);
                        A.active[nxt * A.max_entries + idx] = e;
                    }
                }
            }
            if (!grid_barrier(A.gs, v.status)) return;
            mark(kBtStepDone, na);
            cur = nxt;
        }
        if (!grid_barrier(A.gs, v.status)) return;
        mark(kBtCmdDone, 0);
    }
}

}  // namespace gb
