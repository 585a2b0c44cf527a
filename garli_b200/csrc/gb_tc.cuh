// gb_tc.cuh -- tensor-core CLA update for the 20- and 61-state models
// (precision form, FP32 CLA segment), with exact integer accumulation.
//
// Per rate category r the update is two dense products followed by an
// element-wise one (Tree::CalcFullCLAInternalInternalNState, tree.cpp:7843):
//     dest[p, r, i] = (sum_j P1_r[i][j] L[p, r, j]) * (sum_j P2_r[i][j] R[p, r, j]).
//
// Each product runs on the tensor cores as signed 8-bit digit products with
// 32-bit integer accumulation (tcgen05.mma kind::i8), which is exact: nothing
// is rounded or truncated inside the tensor core.  The operands are split into
// base-256 digits over a per-row power-of-two scale (the scheme of Ootomo,
// Ozaki and Yokota, "DGEMM on integer matrix multiplication unit", 2024):
//   * a child CLA row (pattern p, category r) with max_j L < 2^eA is held as
//     the 38-bit integer round(L 2^(38-eA)): |L - Lq| <= 2^(eA-39);
//   * a row i of P_r with max_j P < 2^eB as round(P 2^(38-eB)):
//     |P - Pq| <= 2^(eB-39);
//   * each integer N is written with five balanced digits d_0..d_4 in
//     [-128, 127] (d_0 most significant): the bytes of N + 0x8080808080, each
//     less 128;
//   * the digit products d_k . e_l with k + l = w are summed into class w
//     (w = 0..4, fifteen products), and the classes are combined in 64-bit
//     integers:  sum_j Pq Lq ~ 2^(eA+eB-44) (C0 2^32 + C1 2^24 + C2 2^16 + C3 2^8 + C4).
//     The dropped classes (k + l >= 5) are sums of products of low-order
//     balanced digits, of either sign: their error has no bias.
// Error bound of one product, absolute, with P's rows summing to at most 1
// (2^eA <= 2 max_j L, 2^eB <= 2):
//     |sum_j P L - computed| <= (2^-38 + 2^-38 S + 2^-34 S) max_j L,
// the terms from L's and P's representation and from the dropped classes:
// 1.2e-9 max_j L for 20 states, 3.7e-9 for 61; the 64-bit sum is converted to
// FP64 once (relative 2^-53).  That is below the FP32 storage of the result
// (relative 2^-24, unbiased stochastic rounding), which stays the dominant
// error of the precision form.  Tip children are not put on the tensor cores:
// their product is a column of P (or a row sum, for missing data) read in FP64.
//
// One CTA per SM (about 200 KB of shared memory) and warp roles:
//   warps 0-3  epilogue: read the class sums back from TMEM (tcgen05.ld),
//              combine, multiply the two children, round stochastically to
//              FP32 into a shared tile; per pattern the power-of-two
//              normalisation and the integer scaler; coalesced stores;
//   warps 4-7  producer: 1-D bulk copies (cp.async.bulk, this GPU's own
//              memory, no multicast) of both children's FP32 tiles into
//              shared memory, row exponents, digit planes in the UMMA
//              K-major layout;
//   warp 8     one thread issues the UMMAs (M = 128 patterns, N = 32 states,
//              K = 32 digits) into a ring of three TMEM regions (5 classes x
//              32 columns each) and commits them to mbarriers.
// Every wait is bounded; a timeout sets a status bit, the roles wind down,
// copies and MMAs in flight are waited for (bounded) and TMEM is freed.
// A pattern whose product maximum is below 2^-64 (FP32 would lose digits of
// its smaller entries) sets kStatusTcRange; the engine then recomputes the
// CLAs on the CUDA cores.
#pragma once
#include "gb_batch_mixed.cuh"
#include "gb_common.cuh"
#include "gb_stage.cuh"

namespace gb {

enum : int { kStatusTcTimeout = 8, kStatusTcRange = 16 };
constexpr int kTcM = 128;                       // patterns per tile (UMMA M)
constexpr int kTcEpiWarps = 4, kTcProdWarps = 4;
constexpr int kTcThreads = 32 * (kTcEpiWarps + kTcProdWarps + 1);
constexpr int kDigA = 5, kDigB = 5, kTcClasses = 5;
constexpr unsigned long long kDigBias = 0x8080808080ULL;  // + 128 in every digit position
constexpr int kTcRegions = 3, kTcRegionCols = kTcClasses * 32;
constexpr int kTcSlots = 2;
constexpr int kBarEpi = 1, kBarProd = 2;        // named barriers (0 is __syncthreads)

// Shapes and shared-memory layout of one CTA.  K (the "to" state j) is padded
// to whole 32-digit UMMA K steps, N (the "from" state i) to 32-state halves.
template <int S, int R>
struct I8Cfg {
    static constexpr int KB = (S + 31) / 32 * 32;  // digit bytes per row
    static constexpr int KSTEPS = KB / 32;
    static constexpr int NH = (S + 31) / 32;
    static constexpr int NPAD = NH * 32;
    static constexpr int RS = R * S;
    static constexpr int RSP = RS | 1;              // odd row stride of the output tile: no bank conflicts
    static constexpr int STAGE = kTcM * RS * 4;     // FP32 tile of one child
    static constexpr int APLANE = kTcM * KB;
    static constexpr int ASLOT = kDigA * APLANE;    // digits of one (child, category)
    static constexpr int BPLANE = NPAD * KB;
    static constexpr int BSET = kDigB * BPLANE;     // digits of one P_r
    static constexpr int SBO = KB * 8;              // bytes between 8-row core-matrix groups
    static constexpr int OFF_STAGE = 0;
    static constexpr int OFF_ASLOT = OFF_STAGE + 2 * STAGE;
    static constexpr int OFF_B = OFF_ASLOT + kTcSlots * ASLOT;
    static constexpr int OFF_OUT = OFF_B + 2 * R * BSET;
    static constexpr int OFF_SB = OFF_OUT + kTcM * RSP * 4;     // double [2][R][NPAD]: 2^(eB - 22)
    static constexpr int OFF_TSUM = OFF_SB + 2 * R * NPAD * 8;  // double [2][R][NPAD]: row sums of P
    static constexpr int OFF_EA = OFF_TSUM + 2 * R * NPAD * 8;  // int [2 tiles][2 children][R][128]
    static constexpr int OFF_ROW = OFF_EA + 2 * 2 * R * kTcM * 4;  // float [128]: 2^-e of each pattern
    static constexpr int BYTES = OFF_ROW + kTcM * 4;
    static_assert(STAGE % 16 == 0 && OFF_ASLOT % 16 == 0 && OFF_B % 16 == 0, "bulk-copy / UMMA alignment");
};

// byte offset of digit (row n, byte k) of a K-major operand with KB bytes
// per row in the canonical no-swizzle layout: 8-row x 16-byte core matrices,
// K-adjacent ones 128 B apart (LBO), 8-row groups KB * 8 B apart (SBO)
__device__ __forceinline__ uint32_t i8_off(int n, int k, int KB) {
    return (uint32_t)(((n >> 3) * (KB >> 4) + (k >> 4)) * 128 + (n & 7) * 16 + (k & 15));
}

// UMMA shared-memory descriptor: start address, LBO, SBO (all >> 4),
// descriptor version 1 (bit 46), base offset 0, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ULL << 46);
}

// instruction descriptor of kind::i8: D = S32 (bits 4-5 = 2), A = B = signed
// 8-bit (format 1, bits 7-9 and 10-12), both K-major, N = 32, M = 128
constexpr uint32_t kI8Idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(kI8Idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t r[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> shared of this CTA, completion counted on mbar
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(mbar)
        : "memory");
}
// named barrier over `n` threads that also agrees on a flag: true only if
// every participant passed true (a role whose wait gave up leaves together)
__device__ __forceinline__ bool group_all(bool ok, int id, int n) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)ok), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// bounded wait that also gives up as soon as another role has given up
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity, volatile int *abort) {
    unsigned long long t0 = 0;
    for (long long it = 0; it < (1LL << 24); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 0) {
            if (*abort) return false;
            const unsigned long long t = stage_ns();
            if (it == 0) t0 = t;
            else if (t - t0 > 2000000000ULL) break;
        }
    }
    *abort = 1;
    return false;
}

// 38-bit fixed point of a non-negative float over 2^eA (value < 2^eA):
// round(x 2^(38 - eA)), from the float's bits (exact shifts, round half up);
// below 2^(eA-39) it is 0
__device__ __forceinline__ unsigned long long fix38(uint32_t bits, int eA) {
    const int e = (int)((bits >> 23) & 0xff);
    if (e == 0) return 0ull;  // zero or subnormal (< 2^-126): far below any row scale in use
    const uint32_t m = (bits & 0x7fffffu) | 0x800000u;  // value = m 2^(e - 150)
    const int sh = e - 112 - eA;                         // N = m 2^sh, sh <= 14: N < 2^38
    if (sh >= 0) return (unsigned long long)m << sh;
    const int s = -sh;
    if (s > 25) return 0ull;
    return (unsigned long long)((m + (1u << (s - 1))) >> s);
}

// exponent eA with max < 2^eA for a row maximum's bits (0 for an all-zero row)
__device__ __forceinline__ int row_exp(uint32_t maxbits) {
    const int e = (int)((maxbits >> 23) & 0xff);
    return e == 0 ? 0 : e - 126;
}

template <int S, int R>
__global__ void __launch_bounds__(kTcThreads, 1) k_cla_i8(View v, LevelOps ops, int tile0, int ntiles) {
    using C = I8Cfg<S, R>;
    extern __shared__ __align__(1024) unsigned char i8_smem[];
    __shared__ __align__(8) unsigned long long s_bar[16];
    __shared__ uint32_t s_taddr;
    __shared__ int s_abort;
    // mbarriers: 0-1 staging full (per child), 2-3 digit slot full, 4-5 slot empty,
    // 6-8 TMEM region full, 9-11 region empty, 12-13 row exponents full, 14-15 empty
    const uint32_t bar0 = smem_u32(&s_bar[0]);
    auto BAR = [&](int k) { return bar0 + 8u * (uint32_t)k; };
    volatile int *abort = &s_abort;
    const DevOp op = ops.op[blockIdx.y];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nint = op.kind == kIntInt ? 2 : op.kind == kIntTip ? 1 : 0;  // internal children: c1 (and c2)
    const int cbuf[2] = {op.c1, op.c2};
    const int cmat[2] = {op.p1, op.p2};
    unsigned char *stage = i8_smem + C::OFF_STAGE;
    unsigned char *aslot = i8_smem + C::OFF_ASLOT;
    unsigned char *bdig = i8_smem + C::OFF_B;
    float *outs = reinterpret_cast<float *>(i8_smem + C::OFF_OUT);
    double *sB = reinterpret_cast<double *>(i8_smem + C::OFF_SB);
    double *tsum = reinterpret_cast<double *>(i8_smem + C::OFF_TSUM);
    int *eAs = reinterpret_cast<int *>(i8_smem + C::OFF_EA);
    float *rowsc = reinterpret_cast<float *>(i8_smem + C::OFF_ROW);

    if (warp == kTcEpiWarps + kTcProdWarps) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int k = 0; k < 2; k++) mbar_init(BAR(k), 1);
        for (int k = 2; k < 6; k++) mbar_init(BAR(k), 1);
        for (int k = 6; k < 9; k++) mbar_init(BAR(k), 1);
        for (int k = 9; k < 12; k++) mbar_init(BAR(k), kTcEpiWarps * 32);
        for (int k = 12; k < 14; k++) mbar_init(BAR(k), 1);
        for (int k = 14; k < 16; k++) mbar_init(BAR(k), kTcEpiWarps * 32);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // per (child, category, row i of P_r): the row's scale 2^(eB - 22) and sum
    // (the product of a tip with missing data), and the digits of internal children
    for (int it = threadIdx.x; it < 2 * R * C::NPAD; it += blockDim.x) {
        const int c = it / (R * C::NPAD), r = (it / C::NPAD) % R, i = it % C::NPAD;
        const double *P = v.mats + (long long)cmat[c] * v.mat_stride + (long long)r * S * S;
        double mx = 0.0, sum = 0.0;
        if (i < S)
            for (int j = 0; j < S; j++) {
                const double x = __ldg(P + i * S + j);
                mx = fmax(mx, x);
                sum += x;
            }
        tsum[it] = sum;
        const int eB = mx > 0.0 ? ilogb(mx) + 1 : 0;
        sB[it] = pow2d(eB - 22);
        if (c >= nint) continue;
        unsigned char *bset = bdig + (c * R + r) * C::BSET;
        const double sc = pow2d(38 - eB);
        for (int j = 0; j < C::KB; j++) {
            unsigned long long q = 0;
            if (i < S && j < S) {
                q = __double2ull_rn(__ldg(P + i * S + j) * sc);
                if (q > 0x3FFFFFFFFFULL) q = 0x3FFFFFFFFFULL;
            }
            const unsigned long long b = (q + kDigBias) ^ kDigBias;  // balanced digits as bytes
            const uint32_t o = i8_off(i, j, C::KB);
#pragma unroll
            for (int l = 0; l < kDigB; l++) bset[l * C::BPLANE + o] = (unsigned char)(b >> (8 * (4 - l)));
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = s_taddr;
    const int ntile_cta = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    auto tile_p0 = [&](int k) { return (tile0 + (int)blockIdx.x + k * (int)gridDim.x) * kTcM; };

    if (warp >= kTcEpiWarps && warp < kTcEpiWarps + kTcProdWarps) {
        // ---------------------------------------------------------------- producer
        const int pt = threadIdx.x - kTcEpiWarps * 32;
        const int pw = warp - kTcEpiWarps;
        constexpr int NP = kTcProdWarps * 32;
        constexpr bool VEC = S % 4 == 0 && C::RS % 4 == 0;  // float4 rows: 16-byte aligned groups
        uint32_t issued = 0, waited[2] = {0, 0}, slot_cnt = 0;
        auto issue = [&](int k) {
            if (k >= ntile_cta) return;
            issued++;
            if (pt != 0) return;
            const int p0 = tile_p0(k);
            for (int c = 0; c < nint; c++) {
                mbar_expect_tx(BAR(c), C::STAGE);
                bulk_g2s(smem_u32(stage + c * C::STAGE), cla_ptr<float>(v, cbuf[c], p0, C::RS), C::STAGE, BAR(c));
            }
        };
        issue(0);
        bool ok = true;
        for (int k = 0; k < ntile_cta && ok; k++) {
            const int ering = k & 1;
            ok = group_all(tc_wait(BAR(14 + ering), ((k >> 1) & 1) ^ 1, abort), kBarProd, NP);
            // row exponents of every (child, category) row of this tile
            for (int c = 0; c < nint && ok; c++) {
                ok = group_all(tc_wait(BAR(c), waited[c] & 1, abort), kBarProd, NP);
                if (!ok) break;
                waited[c]++;
                const float *row = reinterpret_cast<const float *>(stage + c * C::STAGE) + pt * C::RS;
                for (int r = 0; r < R; r++) {
                    uint32_t mx = 0;
                    for (int t = 0; t < S; t++) {  // rotated start: rows at an even stride hit other banks
                        const int j = (t + pt) % S;
                        mx = max(mx, __float_as_uint(row[r * S + j]));
                    }
                    eAs[((ering * 2 + c) * R + r) * kTcM + pt] = row_exp(mx);
                }
            }
            if (!ok) break;
            ok = group_all(true, kBarProd, NP);
            if (pt == 0) mbar_arrive(BAR(12 + ering));
            // digit planes, one (child, category) per slot
            for (int r = 0; r < R && ok; r++) {
                for (int c = 0; c < nint && ok; c++) {
                    const int s = slot_cnt & 1;
                    ok = group_all(tc_wait(BAR(4 + s), ((slot_cnt >> 1) & 1) ^ 1, abort), kBarProd, NP);
                    if (!ok) break;
                    const float *tile = reinterpret_cast<const float *>(stage + c * C::STAGE);
                    const int *eAr = eAs + ((ering * 2 + c) * R + r) * kTcM;
                    unsigned char *dst = aslot + s * C::ASLOT;
                    // one 8-row x 16-byte core matrix per warp and step: lane = (row, 4-byte word)
                    for (int cm = pw; cm < (kTcM / 8) * (C::KB / 16); cm += kTcProdWarps) {
                        const int rg = cm / (C::KB / 16), kc = cm % (C::KB / 16);
                        const int m = rg * 8 + (lane >> 2);
                        const int j0 = kc * 16 + (lane & 3) * 4;
                        const int eA = eAr[m];
                        const float *src = tile + m * C::RS + r * S + j0;
                        unsigned long long q[4] = {0ull, 0ull, 0ull, 0ull};
                        if (VEC) {
                            if (j0 < S) {
                                const float4 f = *reinterpret_cast<const float4 *>(src);
                                q[0] = fix38(__float_as_uint(f.x), eA);
                                q[1] = fix38(__float_as_uint(f.y), eA);
                                q[2] = fix38(__float_as_uint(f.z), eA);
                                q[3] = fix38(__float_as_uint(f.w), eA);
                            }
                        } else {
#pragma unroll
                            for (int t = 0; t < 4; t++)
                                if (j0 + t < S) q[t] = fix38(__float_as_uint(src[t]), eA);
                        }
                        // balanced digits as bytes: digit 0 is byte 4, digits 1-4 bytes 3..0
                        uint32_t lo[4], hi[4];
#pragma unroll
                        for (int t = 0; t < 4; t++) {
                            const unsigned long long b = (q[t] + kDigBias) ^ kDigBias;
                            lo[t] = (uint32_t)b;
                            hi[t] = (uint32_t)(b >> 32);
                        }
                        const uint32_t o = i8_off(m, j0, C::KB);
                        {
                            const uint32_t a = __byte_perm(hi[0], hi[1], 0x40), b = __byte_perm(hi[2], hi[3], 0x40);
                            *reinterpret_cast<uint32_t *>(dst + o) = __byte_perm(a, b, 0x5410);
                        }
#pragma unroll
                        for (int d = 1; d < kDigA; d++) {
                            // byte (4 - d) of each of the four values, packed in order
                            const uint32_t sel = 4 - d;
                            const uint32_t a = __byte_perm(lo[0], lo[1], sel | ((sel + 4) << 4));
                            const uint32_t b = __byte_perm(lo[2], lo[3], sel | ((sel + 4) << 4));
                            *reinterpret_cast<uint32_t *>(dst + d * C::APLANE + o) = __byte_perm(a, b, 0x5410);
                        }
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    ok = group_all(true, kBarProd, NP);
                    if (pt == 0) mbar_arrive(BAR(2 + s));
                    slot_cnt++;
                }
            }
            if (!ok) break;
            // both staging tiles are consumed (every producer thread is past the
            // barrier above): fetch the next tile's children
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(k + 1);
        }
        // copies still in flight are waited for (bounded) before the CTA can exit
        if (pt == 0)
            for (int c = 0; c < nint; c++)
                for (uint32_t n = waited[c]; n < issued; n++) mbar_wait(BAR(c), n & 1);
    } else if (warp == kTcEpiWarps + kTcProdWarps) {
        // ---------------------------------------------------------------- MMA issuer
        if (lane == 0 && nint > 0) {
            uint32_t slot_cnt = 0, unit = 0;
            bool ok = true;
            for (int k = 0; k < ntile_cta && ok; k++) {
                for (int r = 0; r < R && ok; r++) {
                    int slot[2];
                    for (int c = 0; c < nint && ok; c++) {
                        slot[c] = slot_cnt & 1;
                        ok = tc_wait(BAR(2 + slot[c]), (slot_cnt >> 1) & 1, abort);
                        slot_cnt++;
                    }
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    for (int h = 0; h < C::NH && ok; h++) {
                        for (int c = 0; c < nint && ok; c++) {
                            const int q = unit % kTcRegions;
                            ok = tc_wait(BAR(9 + q), ((unit / kTcRegions) & 1) ^ 1, abort);
                            if (!ok) break;
                            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                            const uint32_t d0 = taddr + (uint32_t)(q * kTcRegionCols);
                            const uint32_t abase = smem_u32(aslot + slot[c] * C::ASLOT);
                            const uint32_t bbase = smem_u32(bdig + (c * R + r) * C::BSET) + h * 4 * C::SBO;
#pragma unroll
                            for (int w = 0; w < kTcClasses; w++) {
                                bool first = true;
#pragma unroll
                                for (int ka = 0; ka < kDigA; ka++) {
                                    const int lb = w - ka;
                                    if (lb < 0 || lb >= kDigB) continue;
#pragma unroll
                                    for (int st = 0; st < C::KSTEPS; st++) {
                                        const uint64_t ad = umma_desc(abase + ka * C::APLANE + st * 256, 128, C::SBO);
                                        const uint64_t bd = umma_desc(bbase + lb * C::BPLANE + st * 256, 128, C::SBO);
                                        umma_i8(d0 + w * 32, ad, bd, first ? 0u : 1u);
                                        first = false;
                                    }
                                }
                            }
                            umma_commit(BAR(6 + q));
                            unit++;
                            if (h == C::NH - 1) umma_commit(BAR(4 + slot[c]));
                        }
                    }
                }
            }
            // every MMA issued has completed before TMEM can be freed
            if (unit > 0) {
                const int q = (unit - 1) % kTcRegions;
                mbar_wait(BAR(6 + q), ((unit - 1) / kTcRegions) & 1);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- epilogue
        const int m = threadIdx.x;  // TMEM lane = pattern row of the tile
        const uint32_t trow = taddr + ((uint32_t)(warp * 32) << 16);
        uint32_t unit = 0;
        for (int k = 0; k < ntile_cta; k++) {
            const int p0 = tile_p0(k), p = p0 + m;
            const bool live = p < v.npat;
            const int ering = k & 1;
            if (!group_all(tc_wait(BAR(12 + ering), (k >> 1) & 1, abort), kBarEpi, kTcEpiWarps * 32)) break;
            int code[2] = {S, S};
            for (int c = nint; c < 2; c++)
                if (live) code[c] = v.tips[(long long)cbuf[c] * v.npat_pad + p];
            float *dst_tile = cla_ptr<float>(v, op.dest, p0, C::RS);
            double mx = 0.0;
            bool ok = true;
            for (int r = 0; r < R && ok; r++) {
                double ea[2] = {1.0, 1.0};
                for (int c = 0; c < nint; c++) ea[c] = pow2d(eAs[((ering * 2 + c) * R + r) * kTcM + m] - 22);
                for (int h = 0; h < C::NH && ok; h++) {
                    int q[2] = {0, 0};
                    for (int c = 0; c < nint; c++) {
                        q[c] = unit % kTcRegions;
                        ok = ok && tc_wait(BAR(6 + q[c]), (unit / kTcRegions) & 1, abort);
                        unit++;
                    }
                    // the warp's TMEM reads below are warp-collective: its lanes decide together
                    ok = __all_sync(0xffffffffu, ok);
                    if (!ok) break;
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                    for (int c8 = 0; c8 < 32; c8 += 8) {
                        if (h * 32 + c8 >= S) break;  // uniform across the warp
                        double d[2][8];
                        for (int c = 0; c < 2; c++) {
                            if (c < nint) {
                                uint32_t t[kTcClasses][8];
#pragma unroll
                                for (int w = 0; w < kTcClasses; w++)
                                    tmem_ld8(trow + (uint32_t)(q[c] * kTcRegionCols + w * 32 + c8), t[w]);
                                tmem_wait_ld();
#pragma unroll
                                for (int j = 0; j < 8; j++) {
                                    const long long acc = (long long)(int)t[0][j] * (1ll << 32) +
                                                          (long long)(int)t[1][j] * (1ll << 24) +
                                                          (long long)(int)t[2][j] * (1ll << 16) +
                                                          (long long)(int)t[3][j] * (1ll << 8) + (long long)(int)t[4][j];
                                    const int i = min(h * 32 + c8 + j, C::NPAD - 1);
                                    // the exact product is >= 0; the dropped classes may leave a tiny negative
                                    d[c][j] = fmax(0.0, (double)acc * sB[(c * R + r) * C::NPAD + i] * ea[c]);
                                }
                            } else {
                                const double *P = v.mats + (long long)cmat[c] * v.mat_stride + (long long)r * S * S;
#pragma unroll
                                for (int j = 0; j < 8; j++) {
                                    const int i = h * 32 + c8 + j;
                                    double x = 0.0;
                                    if (i < S)
                                        x = code[c] < S ? __ldg(P + i * S + code[c]) : tsum[(c * R + r) * C::NPAD + i];
                                    d[c][j] = x;
                                }
                            }
                        }
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            const int i = h * 32 + c8 + j;
                            if (i < S) {
                                const double x = d[0][j] * d[1][j];
                                mx = fmax(mx, x);
                                const int idx = r * S + i;
                                const unsigned int key =
                                    (unsigned int)(reinterpret_cast<unsigned long long>(dst_tile + m * C::RS + idx) >> 2);
                                outs[m * C::RSP + idx] = live ? round_stochastic_exact(x, key) : 0.f;
                            }
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    for (int c = 0; c < nint; c++) mbar_arrive(BAR(9 + q[c]));
                }
            }
            mbar_arrive(BAR(14 + ering));
            ok = group_all(ok, kBarEpi, kTcEpiWarps * 32);
            if (!ok) break;
            // power-of-two normalisation of each pattern and its scaler
            int e = 0;
            if (mx > 0.0) e = max(-126, min(126, ilogb(mx)));
            if (live && mx > 0.0 && mx < 5.421010862427522e-20) atomicOr(v.status, kStatusTcRange);  // 2^-64
            rowsc[m] = __int_as_float((127 - e) << 23);
            if (live) {
                int ms = 0;
                if (op.kind != kTipTip) ms += v.scalers[(long long)op.c1 * v.npat_pad + p];
                if (op.kind == kIntInt) ms += v.scalers[(long long)op.c2 * v.npat_pad + p];
                v.scalers[(long long)op.dest * v.npat_pad + p] = ms - e;
            }
            group_all(true, kBarEpi, kTcEpiWarps * 32);
            // coalesced store of the tile (rows beyond the last pattern are skipped)
            const int nrow = min(kTcM, v.npat - p0);
            for (int x = m; x < nrow * C::RS; x += kTcEpiWarps * 32) {
                const int row = x / C::RS, col = x - row * C::RS;
                dst_tile[x] = outs[row * C::RSP + col] * rowsc[row];
            }
            group_all(true, kBarEpi, kTcEpiWarps * 32);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0 && s_abort) atomicOr(v.status, kStatusTcTimeout);
    if (warp == kTcEpiWarps + kTcProdWarps)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(512u));
}

}  // namespace gb
