// gb_tc.cuh -- tensor-core CLA update for the 20- and 61-state models
// (precision form, FP32 CLA segment).
//
// Per rate category r the update is two dense products followed by an
// element-wise one (Tree::CalcFullCLAInternalInternalNState, tree.cpp:7843):
//     dest[p, r, i] = (sum_j P1_r[i][j] L[p, r, j]) * (sum_j P2_r[i][j] R[p, r, j]).
// A CTA takes 128 patterns of one op, one child at a time with as many rate
// categories per round as TMEM holds.  Each product is a 128 x 32 x K UMMA
// per 32-state half (M = patterns, K = states padded to 24 / 64) issued by one
// thread with tcgen05.mma kind::tf32, operands in shared memory (K-major, no
// swizzle), results in TMEM.  Operands are split x = hi + lo with hi = tf32(x),
// lo = tf32(x - hi) (3xTF32): A.B ~ Ahi.Bhi + Ahi.Blo + Alo.Bhi.  The tensor
// core's FP32 accumulation truncates, so the dominant Ahi.Bhi term is never
// accumulated across instructions: every 8-wide K step writes its own TMEM
// region, the regions are summed in FP64 on the CUDA cores, each plus the
// measured mean truncation loss of one instruction (corr_ulps ulp of its
// result) unless the row is exact (a one-hot tip); only the small cross terms
// share an accumulator.  A tip child
// is a one-hot row (all ones when missing), so every op kind is the same
// product.  Products of the two children are kept per pattern in FP64 shared
// memory; the pattern's power-of-two normalisation over all categories and
// states follows, and FP32 stores use unbiased stochastic rounding.
// Every mbarrier wait is bounded; a CTA always frees its TMEM.
#pragma once
#include "gb_batch_mixed.cuh"
#include "gb_common.cuh"

namespace gb {

enum : int { kStatusTcTimeout = 8 };
// mean loss, in ulps of the result, of one tcgen05.mma kind::tf32 result with
// FP32 accumulation (truncating alignment and normalisation), added back to
// every inexact K-step result.  Measured on B200: the lnL bias against the
// FP64 oracle is linear in this value and crosses zero at 0.63-0.70 ulp on the
// 20- and 61-state test and benchmark alignments (0 ulp: -4e-8 relative lnL;
// no correction of the accumulated form: -1.2e-7).
constexpr double kTcCorrUlps = 0.66;
constexpr int kTcM = 128;      // patterns per CTA (UMMA M)
constexpr int kTcThreads = 256;  // two warpgroups: both stage; each reads back half of the TMEM columns

template <int S>
struct TcShape {
    static constexpr int KP = (S + 7) / 8 * 8;     // K padded to the tf32 UMMA K step (8)
    static constexpr int NP = (S + 15) / 16 * 16;  // N padded to a multiple of 16
};

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// byte offset of element (row m, column k) of a K-major operand with KP
// columns in the canonical no-swizzle layout: 8-row x 16-byte core matrices,
// the K-adjacent core matrices 128 B apart (LBO), 8-row groups KP*32 B apart (SBO)
__device__ __forceinline__ uint32_t kmaj_off(int m, int k, int KP) {
    return (uint32_t)(((m >> 3) * (KP >> 2) + (k >> 2)) * 128 + (m & 7) * 16 + (k & 3) * 4);
}

// UMMA shared-memory descriptor: start address, LBO, SBO (all >> 4), version 1,
// base offset 0, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ULL << 46);
}

// instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N
__host__ __device__ constexpr uint32_t tc_idesc(int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_ld8(uint32_t taddr, float v[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tc_ld8_nw(uint32_t taddr, uint32_t r[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// Stage rows [p0, p0 + 128) of one child (CLA or tip) for category r as hi/lo
// tf32 operands, four K-consecutive elements (one 16-byte core-matrix row
// segment) per step; the global loads are float4 when rows are 16-byte aligned.
template <int S, int R>
__device__ __forceinline__ void tc_stage_a(const View &v, int child, bool tip, int p0, int r, unsigned char *hi,
                                           unsigned char *lo) {
    constexpr int KP = TcShape<S>::KP, KQ = KP / 4;
    constexpr bool VEC = (R * S) % 4 == 0 && S % 4 == 0;
    const float *src = tip ? nullptr : cla_ptr<float>(v, child, p0, R * S);
#pragma unroll 2
    for (int idx = threadIdx.x; idx < kTcM * KQ; idx += blockDim.x) {
        const int m = idx / KQ, k0 = (idx % KQ) * 4;
        const int p = p0 + m;
        float x[4] = {0.f, 0.f, 0.f, 0.f};
        if (p < v.npat) {
            if (tip) {
                const int code = v.tips[(long long)child * v.npat_pad + p];
#pragma unroll
                for (int j = 0; j < 4; j++) x[j] = (k0 + j < S && (code >= S || code == k0 + j)) ? 1.f : 0.f;
            } else if (VEC && k0 + 4 <= S) {
                const float4 q = __ldg(reinterpret_cast<const float4 *>(src + (long long)m * R * S + r * S + k0));
                x[0] = q.x;
                x[1] = q.y;
                x[2] = q.z;
                x[3] = q.w;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    if (k0 + j < S) x[j] = __ldg(src + (long long)m * R * S + r * S + k0 + j);
            }
        }
        float h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            h[j] = to_tf32(x[j]);
            l[j] = to_tf32(x[j] - h[j]);
        }
        const uint32_t off = kmaj_off(m, k0, KP);
        *reinterpret_cast<float4 *>(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4 *>(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
    }
}

// Stage P_r (rows = "from" states i as N, columns = "to" states j as K).
template <int S, int R>
__device__ __forceinline__ void tc_stage_b(const View &v, int mat, int r, unsigned char *hi, unsigned char *lo) {
    constexpr int KP = TcShape<S>::KP, NP = TcShape<S>::NP, KQ = KP / 4;
    const double *P = v.mats + (long long)mat * v.mat_stride + (long long)r * S * S;
    for (int idx = threadIdx.x; idx < NP * KQ; idx += blockDim.x) {
        const int n = idx / KQ, k0 = (idx % KQ) * 4;
        float h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float x = (n < S && k0 + j < S) ? (float)__ldg(P + n * S + k0 + j) : 0.f;
            h[j] = to_tf32(x);
            l[j] = to_tf32(x - h[j]);
        }
        const uint32_t off = kmaj_off(n, k0, KP);
        *reinterpret_cast<float4 *>(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4 *>(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
    }
}

template <int S, int R>
struct TcSmem {
    static constexpr int KP = TcShape<S>::KP, NP = TcShape<S>::NP;
    static constexpr int KB = KP / 8;            // K steps
    static constexpr int NH = NP / 32;           // 32-state halves of N
    static constexpr int RCOLS = (KB + 1) * 32;  // TMEM columns of one (category, half): K-step regions + cross terms
    static constexpr int A_BYTES = kTcM * KP * 4, B_BYTES = NP * KP * 4;
    static constexpr int RSP = R * S + 1;  // product row stride (odd: no bank conflicts between rows)
    static constexpr int PROD_BYTES = kTcM * RSP * 8;
    // categories per round.  Measured on B200 (20 states, 4 categories): one
    // category per round at 2 CTAs/SM beats four per round at 1 CTA/SM (4.35 vs
    // 6.37 ms per rescore): the staging and FP64 epilogue around the UMMAs are
    // latency-bound and need the second CTA to hide it.
    static constexpr int RG = 1;
    static constexpr int BYTES = RG * (2 * A_BYTES + 2 * B_BYTES) + PROD_BYTES;
    static constexpr int COLS_USED = RG * RCOLS;
    static constexpr int COLS = COLS_USED <= 32 ? 32 : COLS_USED <= 64 ? 64 : COLS_USED <= 128 ? 128
                                : COLS_USED <= 256 ? 256 : 512;
};

// one ulp of a non-negative float (0 for zero and subnormals)
__device__ __forceinline__ double ulp_f(float f) {
    const int e = (__float_as_int(f) >> 23) & 0xff;
    return e == 0 ? 0.0 : pow2d(e - 127 - 23);
}

// One CTA = 128 patterns [first_tile*128 + blockIdx.x*128, +128) of op blockIdx.y.
// A round = one child, RG categories, one 32-state half: stage, issue, wait,
// read back.
template <int S, int R>
__global__ void __launch_bounds__(kTcThreads, 2) k_cla_tc(View v, LevelOps ops, int first_tile, double corr_ulps) {
    using SM = TcSmem<S, R>;
    constexpr int KP = SM::KP, KB = SM::KB, NH = SM::NH, RG = SM::RG;
    constexpr int GB = 2 * SM::A_BYTES + 2 * SM::B_BYTES;  // staging bytes of one category
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long s_mbar;
    __shared__ uint32_t s_taddr;
    double *prod = reinterpret_cast<double *>(tc_smem + RG * GB);  // [128][RSP]
    const DevOp op = ops.op[blockIdx.y];
    const int p0 = (first_tile + blockIdx.x) * kTcM;
    const int warp = threadIdx.x >> 5;
    const int wg = threadIdx.x >> 7;  // warpgroup: which 8-column chunks it reads back
    const int m = threadIdx.x & 127;  // epilogue row (TMEM lane; warp w reads lanes 32 (w % 4) ..)
    const int p = p0 + m;
    const uint32_t mbar = smem_u32(&s_mbar);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"((uint32_t)SM::COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1u));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = s_taddr;
    const uint32_t trow = taddr + ((uint32_t)((warp & 3) * 32) << 16);
    constexpr uint32_t idesc = tc_idesc(32);
    const uint32_t sbo = KP * 32, lbo = 128;
    bool ok = true;
    uint32_t phase = 0;
    for (int c = 0; c < 2 && ok; c++) {
        const int child = c ? op.c2 : op.c1;
        const bool tip = c ? op.kind != kIntInt : op.kind == kTipTip;
        // a row is exact (no truncation to correct) when it is a one-hot tip state
        bool exact_row = false;
        if (tip && p < v.npat) exact_row = v.tips[(long long)child * v.npat_pad + p] < S;
        for (int r0 = 0; r0 < R && ok; r0 += RG) {
            const int ng = min(RG, R - r0);
            for (int g = 0; g < ng; g++) {
                unsigned char *base = tc_smem + g * GB;
                tc_stage_a<S, R>(v, child, tip, p0, r0 + g, base, base + SM::A_BYTES);
                tc_stage_b<S, R>(v, c ? op.p2 : op.p1, r0 + g, base + 2 * SM::A_BYTES,
                                 base + 2 * SM::A_BYTES + SM::B_BYTES);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int h = 0; h < NH && ok; h++) {
                if (threadIdx.x == 0) {
                    // B rows [32h, 32h+32) = 8-row groups 4h .. 4h+3, each SBO bytes apart
                    const uint32_t hoff = (uint32_t)h * 4 * sbo;
                    for (int g = 0; g < ng; g++) {
                        const uint32_t sa = smem_u32(tc_smem + g * GB);
                        const uint32_t ahb = sa, alb = sa + SM::A_BYTES;
                        const uint32_t bhb = sa + 2 * SM::A_BYTES + hoff, blb = bhb + SM::B_BYTES;
                        const uint32_t dbase = taddr + (uint32_t)(g * SM::RCOLS);
                        for (int kb = 0; kb < KB; kb++) {
                            const uint32_t o = kb * 256;
                            const uint64_t ah = umma_desc(ahb + o, lbo, sbo), al = umma_desc(alb + o, lbo, sbo);
                            const uint64_t bh = umma_desc(bhb + o, lbo, sbo), bl = umma_desc(blb + o, lbo, sbo);
                            tc_mma(dbase + kb * 32, ah, bh, idesc, 0);       // main term, own region
                            tc_mma(dbase + KB * 32, ah, bl, idesc, kb > 0);  // cross terms, accumulated
                            tc_mma(dbase + KB * 32, al, bh, idesc, 1);
                        }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                                 : "memory");
                }
                ok = mbar_wait(mbar, phase & 1);
                phase++;
                ok = __syncthreads_and(ok) != 0;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (!ok) break;
                // (P_c V_c)_s for s in [32h, 32h+32): FP64 sum of the K-step regions
                for (int g = 0; g < ng; g++) {
                    const uint32_t rbase = trow + (uint32_t)(g * SM::RCOLS);
                    const int r = r0 + g;
                    for (int c8 = wg * 8; c8 < 32; c8 += 16) {
                        uint32_t t[KB + 1][8];
#pragma unroll
                        for (int kb = 0; kb <= KB; kb++) tc_ld8_nw(rbase + kb * 32 + c8, t[kb]);
                        tc_wait_ld();
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            double val = (double)__uint_as_float(t[KB][j]);
#pragma unroll
                            for (int kb = 0; kb < KB; kb++) {
                                const float f = __uint_as_float(t[kb][j]);
                                val += (double)f + (exact_row ? 0.0 : corr_ulps * ulp_f(f));
                            }
                            const int st = h * 32 + c8 + j;
                            if (st < S) {
                                double *q = prod + (long long)m * SM::RSP + r * S + st;
                                *q = c ? *q * val : val;
                            }
                        }
                    }
                }
                // the next round's MMAs overwrite TMEM and shared memory: every read above is complete
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncthreads();
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            }
        }
    }
    if (!ok) {
        if (threadIdx.x == 0) atomicOr(v.status, kStatusTcTimeout);
    } else {
        // row m: each warpgroup takes half of the R*S entries; the row max is combined in shared
        // memory (the staging area, free once the last products are read back)
        double(*s_mx)[kTcM] = reinterpret_cast<double(*)[kTcM]>(tc_smem);
        const double *row = prod + (long long)m * SM::RSP;
        const int k0 = wg ? (R * S) / 2 : 0, k1 = wg ? R * S : (R * S) / 2;
        double mx = 0.0;
        for (int k = k0; k < k1; k++) mx = fmax(mx, row[k]);
        s_mx[wg][m] = mx;
        __syncthreads();
        mx = fmax(s_mx[0][m], s_mx[1][m]);
        if (p < v.npat) {
            int e = 0;
            if (mx > 0.0) e = max(-1000, min(1000, ilogb(mx)));
            const double sc = pow2d(-e);
            float *dst = cla_ptr<float>(v, op.dest, p, R * S);
            for (int k = k0; k < k1; k++)
                dst[k] = round_stochastic_exact(row[k] * sc,
                                                (unsigned int)(reinterpret_cast<unsigned long long>(dst + k) >> 2));
            if (wg == 0) {
                int ms = 0;
                if (op.kind != kTipTip) ms += v.scalers[(long long)op.c1 * v.npat_pad + p];
                if (op.kind == kIntInt) ms += v.scalers[(long long)op.c2 * v.npat_pad + p];
                v.scalers[(long long)op.dest * v.npat_pad + p] = ms - e;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"((uint32_t)SM::COLS));
}

}  // namespace gb
