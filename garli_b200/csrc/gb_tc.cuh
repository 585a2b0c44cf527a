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
// FP64 exactly.  That is below the FP32 storage of the result (relative
// 2^-24, unbiased stochastic rounding), which stays the dominant error of the
// precision form.  Tip children are not put on the tensor cores: their
// product is a column of P (or a row sum, for missing data) read in FP64.
//
// One CTA per SM (up to about 220 KB of shared memory) and warp roles:
//   warps 0-7  epilogue, two warps per TMEM lane quadrant (each takes every
//              other 4-state chunk): read the class sums back from TMEM
//              (tcgen05.ld), combine them, multiply the two children, scale
//              by the pattern's power of two and round stochastically to
//              FP32; 16-byte stores straight to the destination CLA (or, for
//              rows that are not 16-byte multiples, a shared tile written
//              out by one bulk copy);
//   warps 8-15 producer: 1-D bulk copies (cp.async.bulk, this GPU's own
//              memory, no multicast) of both children's FP32 tiles into
//              shared memory, row exponents, digit planes in the UMMA
//              K-major layout;
//   warp 16    one thread issues the UMMAs (M = 128 patterns, N = 32 states,
//              K = 32 digits) into a ring of three TMEM regions (5 classes x
//              32 columns each) and commits them to mbarriers.
// The pattern's power of two is fixed before its products are formed: the
// children's row exponents bound every product, (P1 L)(P2 R) <= 2^(E1+E2)
// with E_c the largest row exponent of child c over the categories (0 for a
// tip), so the stored CLA is at most 1 and its scaler is the children's less
// E1 + E2.  The next update rescales from its own row maxima.
// Every wait is bounded; a timeout sets a status bit, the roles wind down,
// copies and MMAs in flight are waited for (bounded) and TMEM is freed.
// A pattern whose largest scaled product is below 2^-64 (FP32 would lose
// digits of its smaller entries) sets kStatusTcRange; the engine then
// recomputes the CLAs on the CUDA cores.
#pragma once
#include "gb_batch_mixed.cuh"
#include "gb_common.cuh"
#include "gb_stage.cuh"

namespace gb {

enum : int { kStatusTcTimeout = 8, kStatusTcRange = 16 };
constexpr int kTcM = 128;                         // patterns per tile (UMMA M)
constexpr int kTcEpiWarps = 8, kTcProdWarps = 8;  // two epilogue warps per TMEM lane quadrant
constexpr int kTcMmaWarp = kTcEpiWarps + kTcProdWarps;
constexpr int kTcThreads = 32 * (kTcMmaWarp + 1);
constexpr int kTcEpi = 32 * kTcEpiWarps, kTcProd = 32 * kTcProdWarps;
constexpr int kDigA = 5, kDigB = 5, kTcClasses = 5;
constexpr unsigned long long kDigBias = 0x8080808080ULL;  // + 128 in every digit position
constexpr int kTcRegions = 3, kTcRegionCols = kTcClasses * 32;
constexpr int kTcSlots = 2;
constexpr int kBarEpi = 1, kBarProd = 2;  // named barriers (0 is __syncthreads)

// Shapes and shared-memory layout of one CTA.  K (the "to" state j) is padded
// to whole 32-digit UMMA K steps, N (the "from" state i) to 32-state halves.
template <int S, int R>
struct I8Cfg {
    static constexpr int KB = (S + 31) / 32 * 32;  // digit bytes per row
    static constexpr int KSTEPS = KB / 32;
    static constexpr int NH = (S + 31) / 32;
    static constexpr int NPAD = NH * 32;
    static constexpr int RS = R * S;
    static constexpr int G = (S + 3) / 4;           // 4-element groups of a row holding data
    static constexpr bool DIRECT = S % 4 == 0;      // 4-state chunks are 16-byte aligned in the CLA
    static constexpr int STAGE = kTcM * RS * 4;     // FP32 tile of one child
    static constexpr int APLANE = kTcM * KB;
    static constexpr int ASLOT = kDigA * APLANE;    // digits of one (child, category)
    static constexpr int BPLANE = NPAD * KB;
    static constexpr int BSET = kDigB * BPLANE;     // digits of one P_r
    static constexpr int SBO = KB * 8;              // bytes between 8-row core-matrix groups
    static constexpr int OUT = DIRECT ? 0 : STAGE;  // output tile for the bulk store
    static constexpr int OFF_STAGE = 0;
    static constexpr int OFF_ASLOT = OFF_STAGE + 2 * STAGE;
    // the op's tables, one contiguous block (written by k_pdigits, one bulk copy per CTA):
    static constexpr int OFF_B = OFF_ASLOT + kTcSlots * ASLOT;    // digits of P_r, [2][R] sets
    static constexpr int OFF_SB = OFF_B + 2 * R * BSET;           // double [2][R][NPAD]: 2^(eB - 22)
    static constexpr int OFF_NMSB = OFF_SB + 2 * R * NPAD * 8;    // double [2][R][NPAD]: -1.5 2^52 2^(eB - 22)
    static constexpr int OFF_TSUM = OFF_NMSB + 2 * R * NPAD * 8;  // double [2][R][NPAD]: row sums of P
    static constexpr int OPB = OFF_TSUM + 2 * R * NPAD * 8 - OFF_B;  // bytes of one op's tables
    static constexpr int OFF_OUT = OFF_B + OPB;
    static constexpr int OFF_EA = OFF_OUT + OUT;                  // int [2 tiles][2 children][R][128]
    static constexpr int OFF_MX = OFF_EA + 2 * 2 * R * kTcM * 4;  // double [2][128]: each half's largest product
    static constexpr int BYTES = OFF_MX + 2 * kTcM * 8;
    static_assert(STAGE % 16 == 0 && OFF_ASLOT % 16 == 0 && OFF_B % 16 == 0 && OFF_OUT % 16 == 0 &&
                      OPB % 16 == 0,
                  "bulk-copy / UMMA alignment");
    static_assert(DIRECT || RS % 2 == 1, "a shared output tile needs an odd row stride (no bank conflicts)");
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
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t r[4]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }
// 1-D bulk copy shared -> global (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_s2g(void *dst, uint32_t src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

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

// bounded wait that also gives up as soon as another role has given up.  Each
// try_wait suspends the thread until the phase completes or 20 microseconds
// pass (a waiting warp takes no issue slots from the warps doing the work);
// after about two seconds the wait gives up and raises the abort flag.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity, volatile int *abort) {
    const unsigned long long t0 = stage_ns();
    for (int it = 0; it < (1 << 20); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity), "r"(20000u)
            : "memory");
        if (done) return true;
        if (*abort) return false;
        if (stage_ns() - t0 > 2000000000ULL) break;
    }
    *abort = 1;
    return false;
}

// 38-bit fixed point of a non-negative float over 2^eA (value < 2^eA):
// round(x 2^(38 - eA)) from the float's bits: the significand shifted left by
// the exponent difference plus 25 (at most 39: below 2^63), then rounded half
// up over those 25 bits; values below 2^(eA - 64) come out 0
__device__ __forceinline__ unsigned long long fix38(uint32_t bits, int eA) {
    const uint32_t e = (bits >> 23) & 0xffu;
    const uint32_t m = e ? ((bits & 0x7fffffu) | 0x800000u) : 0u;  // value = m 2^(e - 150)
    const int sh = max((int)e - 87 - eA, 0);                        // (e - 112 - eA) + 25
    return (((unsigned long long)m << sh) + (1ull << 24)) >> 25;
}

// exponent eA with max < 2^eA for a row maximum's bits (0 for an all-zero row)
__device__ __forceinline__ int row_exp(uint32_t maxbits) {
    const int e = (int)((maxbits >> 23) & 0xff);
    return e == 0 ? 0 : e - 126;
}

// Unbiased stochastic rounding of a non-negative double to float: a uniform
// 29-bit integer is added below the float's last place of the double's bit
// pattern and the 29 bits are cut (the carry moves the value up with
// probability equal to the cut fraction).  Exact for values in the float's
// normal range; values below 2^-126 give 0.
__device__ __forceinline__ float round_stochastic_bits(double x, uint32_t u) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x) + (u >> 3);
    const uint32_t f = (uint32_t)(b >> 29) - (896u << 23);
    return x >= 1.1754943508222875e-38 ? __uint_as_float(f) : 0.0f;
}
// 32-bit linear congruential generator (Numerical Recipes constants); its
// upper bits drive the stochastic rounding
__device__ __forceinline__ uint32_t lcg32(uint32_t &s) {
    s = s * 1664525u + 1013904223u;
    return s;
}

// Per op of a level: the tables every CTA of that op needs, in the CTA's
// shared-memory layout -- per (child, category, row i of P_r) the row's scale
// 2^(eB - 22), -1.5 2^52 times it (the exact int64 -> FP64 rescale of the
// epilogue) and the row sum (the product of a tip with missing data), and for
// internal children the five digit planes of P_r.  One CTA per op.
template <int S, int R>
__global__ void __launch_bounds__(kThreads) k_pdigits(View v, LevelOps ops, unsigned char *out) {
    using C = I8Cfg<S, R>;
    __shared__ int s_eB[2 * R * C::NPAD];
    const DevOp op = ops.op[blockIdx.x];
    const int nint = op.kind == kIntInt ? 2 : op.kind == kIntTip ? 1 : 0;
    const int cmat[2] = {op.p1, op.p2};
    unsigned char *base = out + (long long)blockIdx.x * C::OPB;
    double *sB = reinterpret_cast<double *>(base + (C::OFF_SB - C::OFF_B));
    double *nmsB = reinterpret_cast<double *>(base + (C::OFF_NMSB - C::OFF_B));
    double *tsum = reinterpret_cast<double *>(base + (C::OFF_TSUM - C::OFF_B));
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
        const int eB = mx > 0.0 ? ilogb(mx) + 1 : 0;
        s_eB[it] = eB;
        tsum[it] = sum;
        sB[it] = pow2d(eB - 22);
        nmsB[it] = -6755399441055744.0 * pow2d(eB - 22);  // -1.5 2^52 2^(eB - 22)
    }
    __syncthreads();
    // digits, four consecutive j of one row i per item: one 32-bit word per plane
    constexpr int GK = C::KB / 4;
    for (int it = threadIdx.x; it < nint * R * C::NPAD * GK; it += blockDim.x) {
        const int row = it / GK, g = it % GK;  // row = (c * R + r) * NPAD + i
        const int c = row / (R * C::NPAD), r = (row / C::NPAD) % R, i = row % C::NPAD;
        const double *P = v.mats + (long long)cmat[c] * v.mat_stride + (long long)r * S * S;
        const double sc = pow2d(38 - s_eB[row]);
        uint32_t lo[4], hi[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const int j = 4 * g + t;
            unsigned long long q = 0;
            if (i < S && j < S) {
                q = __double2ull_rn(__ldg(P + i * S + j) * sc);
                if (q > 0x3FFFFFFFFFULL) q = 0x3FFFFFFFFFULL;
            }
            const unsigned long long b = (q + kDigBias) ^ kDigBias;  // balanced digits as bytes
            lo[t] = (uint32_t)b;
            hi[t] = (uint32_t)(b >> 32);
        }
        unsigned char *bset = base + (c * R + r) * C::BSET;
        const uint32_t o = i8_off(i, 4 * g, C::KB);
        *reinterpret_cast<uint32_t *>(bset + o) =
            __byte_perm(__byte_perm(hi[0], hi[1], 0x40), __byte_perm(hi[2], hi[3], 0x40), 0x5410);
#pragma unroll
        for (int d = 1; d < kDigB; d++) {
            const uint32_t sel = (uint32_t)(4 - d) | ((uint32_t)(8 - d) << 4);
            *reinterpret_cast<uint32_t *>(bset + d * C::BPLANE + o) =
                __byte_perm(__byte_perm(lo[0], lo[1], sel), __byte_perm(lo[2], lo[3], sel), 0x5410);
        }
    }
}

template <int S, int R>
__global__ void __launch_bounds__(kTcThreads, 1) k_cla_i8(View v, LevelOps ops, int tile0, int ntiles,
                                                          const unsigned char *pdig) {
    using C = I8Cfg<S, R>;
    extern __shared__ __align__(1024) unsigned char i8_smem[];
    __shared__ __align__(8) unsigned long long s_bar[17];
    __shared__ uint32_t s_taddr;
    __shared__ int s_abort;
    // mbarriers: 0-1 staging full (per child), 2-3 digit slot full, 4-5 slot empty,
    // 6-8 TMEM region full, 9-11 region empty, 12-13 row exponents full, 14-15 empty,
    // 16 the op's tables copied in
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
    double *nmsB = reinterpret_cast<double *>(i8_smem + C::OFF_NMSB);
    double *tsum = reinterpret_cast<double *>(i8_smem + C::OFF_TSUM);
    int *eAs = reinterpret_cast<int *>(i8_smem + C::OFF_EA);
    double *mxs = reinterpret_cast<double *>(i8_smem + C::OFF_MX);

    if (warp == kTcMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int k = 0; k < 9; k++) mbar_init(BAR(k), 1);
        for (int k = 9; k < 12; k++) mbar_init(BAR(k), kTcEpi);
        for (int k = 12; k < 14; k++) mbar_init(BAR(k), 1);
        for (int k = 14; k < 16; k++) mbar_init(BAR(k), kTcEpi);
        mbar_init(BAR(16), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the digit slots' K padding stays zero: conversions write only groups that hold data
    for (int x = threadIdx.x; x < kTcSlots * C::ASLOT / 16; x += blockDim.x)
        reinterpret_cast<uint4 *>(aslot)[x] = make_uint4(0u, 0u, 0u, 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = s_taddr;
    // the op's P digits and scale tables (k_pdigits), one bulk copy from L2
    if (threadIdx.x == 0) {
        mbar_expect_tx(BAR(16), C::OPB);
        bulk_g2s(smem_u32(bdig), pdig + (long long)blockIdx.y * C::OPB, C::OPB, BAR(16));
    }
    const int ntile_cta = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    auto tile_p0 = [&](int k) { return (tile0 + (int)blockIdx.x + k * (int)gridDim.x) * kTcM; };

    if (warp >= kTcEpiWarps && warp < kTcMmaWarp) {
        // ---------------------------------------------------------------- producer
        const int pt = threadIdx.x - kTcEpi;
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
            ok = group_all(tc_wait(BAR(14 + ering), ((k >> 1) & 1) ^ 1, abort), kBarProd, kTcProd);
            for (int c = 0; c < nint && ok; c++) {
                ok = group_all(tc_wait(BAR(c), waited[c] & 1, abort), kBarProd, kTcProd);
                if (ok) waited[c]++;
            }
            if (!ok) break;
            // row exponents of every (child, category) row of this tile: thread = (child, row)
            if (pt < nint * kTcM) {
                const int c = pt / kTcM, m = pt % kTcM;
                const float *row = reinterpret_cast<const float *>(stage + c * C::STAGE) + m * C::RS;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    uint32_t mx = 0;
                    if (C::DIRECT) {
#pragma unroll
                        for (int t = 0; t < S / 4; t++) {  // rotated start: rows at an even stride hit other banks
                            const uint4 q = *reinterpret_cast<const uint4 *>(row + r * S + 4 * ((t + m) % (S / 4)));
                            mx = max(mx, max(max(q.x, q.y), max(q.z, q.w)));
                        }
                    } else {
                        for (int j = 0; j < S; j++) mx = max(mx, __float_as_uint(row[r * S + j]));
                    }
                    eAs[((ering * 2 + c) * R + r) * kTcM + m] = row_exp(mx);
                }
            }
            ok = group_all(true, kBarProd, kTcProd);
            if (pt == 0) mbar_arrive(BAR(12 + ering));
            // digit planes, one (child, category) per slot; thread = (row, 4-element group)
            for (int r = 0; r < R && ok; r++) {
                for (int c = 0; c < nint && ok; c++) {
                    const int s = slot_cnt & 1;
                    ok = group_all(tc_wait(BAR(4 + s), ((slot_cnt >> 1) & 1) ^ 1, abort), kBarProd, kTcProd);
                    if (!ok) break;
                    // two threads per row, each every other 4-element group
                    const int m = pt >> 1;
                    const int eA = eAs[((ering * 2 + c) * R + r) * kTcM + m];
                    const float *src = reinterpret_cast<const float *>(stage + c * C::STAGE) + m * C::RS + r * S;
                    unsigned char *dst = aslot + s * C::ASLOT + i8_off(m, 0, C::KB);
#pragma unroll 2
                    for (int g = pt & 1; g < C::G; g += 2) {
                        const int j0 = 4 * g;
                        unsigned long long q[4];
                        if (C::DIRECT) {
                            const uint4 f = *reinterpret_cast<const uint4 *>(src + j0);
                            q[0] = fix38(f.x, eA);
                            q[1] = fix38(f.y, eA);
                            q[2] = fix38(f.z, eA);
                            q[3] = fix38(f.w, eA);
                        } else {
#pragma unroll
                            for (int t = 0; t < 4; t++)
                                q[t] = j0 + t < S ? fix38(__float_as_uint(src[j0 + t]), eA) : 0ull;
                        }
                        // balanced digits as bytes: digit 0 is byte 4, digits 1-4 bytes 3..0
                        uint32_t lo[4], hi[4];
#pragma unroll
                        for (int t = 0; t < 4; t++) {
                            const unsigned long long b = q[t] + kDigBias;
                            lo[t] = (uint32_t)b;
                            hi[t] = (uint32_t)(b >> 32);
                        }
                        unsigned char *o = dst + (j0 >> 4) * 128 + (j0 & 15);
                        *reinterpret_cast<uint32_t *>(o) =
                            __byte_perm(__byte_perm(hi[0], hi[1], 0x40), __byte_perm(hi[2], hi[3], 0x40), 0x5410) ^
                            0x80808080u;
#pragma unroll
                        for (int d = 1; d < kDigA; d++) {
                            // byte (4 - d) of each of the four values, packed in order
                            const uint32_t sel = (uint32_t)(4 - d) | ((uint32_t)(8 - d) << 4);
                            *reinterpret_cast<uint32_t *>(o + d * C::APLANE) =
                                __byte_perm(__byte_perm(lo[0], lo[1], sel), __byte_perm(lo[2], lo[3], sel), 0x5410) ^
                                0x80808080u;
                        }
                    }
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    ok = group_all(true, kBarProd, kTcProd);
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
        if (pt == 0) {
            for (int c = 0; c < nint; c++)
                for (uint32_t n = waited[c]; n < issued; n++) mbar_wait(BAR(c), n & 1);
            mbar_wait(BAR(16), 0);  // the tables' copy (thread 0 issued it)
        }
    } else if (warp == kTcMmaWarp) {
        // ---------------------------------------------------------------- MMA issuer
        if (lane == 0 && nint > 0) {
            uint32_t slot_cnt = 0, unit = 0;
            bool ok = tc_wait(BAR(16), 0, abort);
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
        const int quad = warp & 3, eh = warp >> 2;  // TMEM lane quadrant; which 4-state chunks
        const int m = quad * 32 + lane;             // TMEM lane = pattern row of the tile
        const uint32_t trow = taddr + ((uint32_t)(quad * 32) << 16);
        uint32_t unit = 0;
        const bool tables = group_all(tc_wait(BAR(16), 0, abort), kBarEpi, kTcEpi);
        for (int k = 0; k < ntile_cta && tables; k++) {
            const int p0 = tile_p0(k), p = p0 + m;
            const bool live = p < v.npat;
            const int ering = k & 1;
            // the previous tile's bulk store has read the output tile before the barrier below
            if (!C::DIRECT && threadIdx.x == 0) bulk_wait_read();
            if (!group_all(tc_wait(BAR(12 + ering), (k >> 1) & 1, abort), kBarEpi, kTcEpi)) break;
            int code[2] = {S, S};
            for (int c = nint; c < 2; c++)
                if (live) code[c] = v.tips[(long long)cbuf[c] * v.npat_pad + p];
            // the pattern's power of two: E1 + E2 bounds every product
            int ecap = 0;
            for (int c = 0; c < nint; c++) {
                int e = -1000;
#pragma unroll
                for (int r = 0; r < R; r++) e = max(e, eAs[((ering * 2 + c) * R + r) * kTcM + m]);
                ecap += e;
            }
            if (eh == 0 && live) {
                int ms = 0;
                if (op.kind != kTipTip) ms += v.scalers[(long long)op.c1 * v.npat_pad + p];
                if (op.kind == kIntInt) ms += v.scalers[(long long)op.c2 * v.npat_pad + p];
                v.scalers[(long long)op.dest * v.npat_pad + p] = ms - ecap;
            }
            float *dst_row = cla_ptr<float>(v, op.dest, p0, C::RS) + m * C::RS;
            uint32_t rng = ((uint32_t)p * 0x9E3779B1u) ^ ((uint32_t)op.dest * 0x85EBCA77u) ^ (eh ? 0xC2B2AE3Du : 0u);
            rng ^= rng >> 16;
            double mx = 0.0;
            bool ok = true;
            for (int r = 0; r < R && ok; r++) {
                int esum = -ecap;
                for (int c = 0; c < nint; c++) esum += eAs[((ering * 2 + c) * R + r) * kTcM + m] - 22;
                const double ea = pow2d(max(esum, -1000));
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
                    const int ncol = min(32, S - h * 32);
                    for (int c4 = eh; 4 * c4 < ncol; c4 += 2) {  // uniform across the warp
                        double d[2][4];
#pragma unroll
                        for (int c = 0; c < 2; c++) {
                            if (c < nint) {
                                uint32_t t[kTcClasses][4];
#pragma unroll
                                for (int w = 0; w < kTcClasses; w++)
                                    tmem_ld4(trow + (uint32_t)(q[c] * kTcRegionCols + w * 32 + 4 * c4), t[w]);
                                tmem_wait_ld();
#pragma unroll
                                for (int j = 0; j < 4; j++) {
                                    long long acc = (long long)(int)t[4][j];
                                    acc += (long long)(int)t[3][j] * 256ll;
                                    acc += (long long)(int)t[2][j] * 65536ll;
                                    acc += (long long)(int)t[1][j] * 16777216ll;
                                    acc += (long long)(int)t[0][j] * 4294967296ll;
                                    // |acc| < 2^51: 1.5 2^52 + acc is exact, and so is the fused rescale
                                    const double dm = __longlong_as_double(acc + 0x4338000000000000ll);
                                    const int ci = (c * R + r) * C::NPAD + min(h * 32 + 4 * c4 + j, C::NPAD - 1);
                                    d[c][j] = fma(dm, sB[ci], nmsB[ci]);
                                }
                            } else {
                                const double *P = v.mats + (long long)cmat[c] * v.mat_stride + (long long)r * S * S;
#pragma unroll
                                for (int j = 0; j < 4; j++) {
                                    const int i = h * 32 + 4 * c4 + j;
                                    double x = 0.0;
                                    if (i < S)
                                        x = code[c] < S ? __ldg(P + i * S + code[c])
                                                        : tsum[(c * R + r) * C::NPAD + i];
                                    d[c][j] = x;
                                }
                            }
                        }
                        float o[4];
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            // the exact product is >= 0; a tiny negative left by the dropped digit
                            // classes rounds to 0 (below the float range)
                            const double x = d[0][j] * d[1][j] * ea;
                            mx = fmax(mx, x);
                            o[j] = round_stochastic_bits(x, lcg32(rng));
                        }
                        const int idx = r * S + h * 32 + 4 * c4;
                        if (C::DIRECT) {
                            if (live) *reinterpret_cast<float4 *>(dst_row + idx) = make_float4(o[0], o[1], o[2], o[3]);
                        } else {
#pragma unroll
                            for (int j = 0; j < 4; j++)
                                if (h * 32 + 4 * c4 + j < S) outs[m * C::RS + idx + j] = live ? o[j] : 0.f;
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    for (int c = 0; c < nint; c++) mbar_arrive(BAR(9 + q[c]));
                }
            }
            mbar_arrive(BAR(14 + ering));
            mxs[eh * kTcM + m] = mx;
            ok = group_all(ok, kBarEpi, kTcEpi);
            if (!ok) break;
            if (eh == 0 && live) {
                const double rmx = fmax(mx, mxs[kTcM + m]);
                if (rmx > 0.0 && rmx < 5.421010862427522e-20) atomicOr(v.status, kStatusTcRange);  // 2^-64
            }
            if (!C::DIRECT) {
                // the output tile is complete (the barrier above): one bulk store
                if (threadIdx.x == 0) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    bulk_s2g(cla_ptr<float>(v, op.dest, p0, C::RS), smem_u32(outs), C::STAGE);
                }
            }
        }
        if (!C::DIRECT && threadIdx.x == 0) bulk_wait_all();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (threadIdx.x == 0 && s_abort) atomicOr(v.status, kStatusTcTimeout);
    if (warp == kTcMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(512u));
}

}  // namespace gb
