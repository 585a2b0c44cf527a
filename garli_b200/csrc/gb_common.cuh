// gb_common.cuh -- shared device-side definitions of the garli_b200 engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gb {

constexpr int kRescaleTableLen = 90;  // RESCALE_ARRAY_LENGTH, tree.h:48
constexpr int kMaxLevelOps = 96;      // CLA ops per batched launch (kernel-parameter bound)
constexpr int kMaxScoreBlocks = 4096; // partial-sum slots for the edge reduction
constexpr int kThreads = 256;

enum OpKind : int { kIntInt = 0, kIntTip = 1, kTipTip = 2 };
enum StatusBits : int { kStatusRescaleRetry = 1, kStatusNonFinite = 2 };

// One CLA update after host normalisation: c1 is the internal child whenever
// exactly one child is a tip (Tree::UpdateCLAs, tree.cpp:3905-3990, swaps the
// children the same way when calling CalcFullCLAInternalTerminal).
struct DevOp {
    int dest, c1, p1, c2, p2;
    int kind;
    int rescale;  // plain form: rank >= rescaleEvery (tree.cpp:3991)
    int wide;     // precision-form batched pass: FP64 buffers, bit 0 dest, bit 1 c1, bit 2 c2
};

enum WideBits : int { kWideDest = 1, kWideC1 = 2, kWideC2 = 4 };

struct LevelOps {
    int n;
    DevOp op[kMaxLevelOps];
};

// Device view of an instance, passed by value to every kernel.
// A CLA buffer holds its first `kpad` patterns in FP64 and the rest in FP32
// (kpad = all patterns in the plain form; in the precision form the patterns
// with large counts, placed first by the instance's internal permutation).
struct View {
    char *partials;           // nbuf x cla_bytes
    int *scalers;             // nbuf x npat_pad
    const uint8_t *tips;      // ntip x npat_pad
    const double *mats;       // nmat x mat_stride: [P | dP | d2P], each R*S*S
    const int *counts;        // npat_pad (0 in the padding)
    const int *const_states;  // npat_pad; -1 = not a constant pattern
    const double *freqs;      // S
    const double *rate_probs; // R
    int *status;
    double *block_sums;       // kMaxScoreBlocks x 3
    double *site_lnl;         // npat_pad
    double *site_d1, *site_d2; // npat_pad each: per-site d lnL / dt, d2 lnL / dt2 of a derivative evaluation
    long long cla_bytes;      // bytes per CLA buffer
    long long mat_stride;     // 3 * R * S * S
    int npat, npat_pad, ntip, kpad, has_pinv, rescale_every;
    double pinv;
};

// Pointer to the R*S slice of pattern p in CLA buffer b (ST must match p's segment).
template <typename ST>
__device__ __forceinline__ ST *cla_ptr(const View &v, int b, int p, int RS);
template <>
__device__ __forceinline__ double *cla_ptr<double>(const View &v, int b, int p, int RS) {
    return reinterpret_cast<double *>(v.partials + (long long)b * v.cla_bytes) + (long long)p * RS;
}
template <>
__device__ __forceinline__ float *cla_ptr<float>(const View &v, int b, int p, int RS) {
    return reinterpret_cast<float *>(v.partials + (long long)b * v.cla_bytes + (long long)v.kpad * RS * 8) +
           (long long)(p - v.kpad) * RS;
}
// 2^k as a double, k in [-1022, 1023]
__device__ __forceinline__ double pow2d(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// ---- 4-state precision form: FP32 elements with an 8-bit mantissa extension ----
// An element x >= 0 of the FP32 segment is the double x cut to 32 significant
// bits: a float word hi (sign, 8-bit exponent, the top 23 mantissa bits) and
// one extension byte e (the next 8), the 21 bits below rounded stochastically
// into the 32 (unbiased to 2^-16 of their unit, the variate a hash of the
// element's place in the pool: the same rounding in every run).  The float
// word alone is x rounded toward zero to FP32.  Encoding and decoding are
// integer operations on the IEEE bit fields: the representation error is
// below 2^-31 x in 5 bytes an element (FP64: 8).  x below 2^-126 (FP32's
// normal range; the pattern's largest element is in [1, 2)) is stored as 0.
// The bytes of a (pattern, category) slice form one 32-bit word (byte k =
// state k); the words follow the FP32 segment in each buffer, R per pattern.
__device__ __forceinline__ unsigned int *cla_ext(const View &v, int b, int p, int RS) {
    return reinterpret_cast<unsigned int *>(v.partials + (long long)b * v.cla_bytes + (long long)v.kpad * RS * 8 +
                                            (long long)(v.npat_pad - v.kpad) * RS * 4) +
           (long long)(p - v.kpad) * (RS / 4);
}
__device__ __forceinline__ double ext_value(float hi, unsigned int e) {
    const unsigned int w = __float_as_uint(hi);
    const unsigned long long E = (w >> 23) & 0xffu;
    const unsigned long long b = ((E + 896ull) << 52) | ((unsigned long long)(w & 0x7fffffu) << 29) |
                                 ((unsigned long long)(e & 0xffu) << 21);
    return E ? __longlong_as_double((long long)b) : 0.0;
}
__device__ __forceinline__ void ext_decode4(const float4 a, unsigned int e, double c[4]) {
    c[0] = ext_value(a.x, e);
    c[1] = ext_value(a.y, e >> 8);
    c[2] = ext_value(a.z, e >> 16);
    c[3] = ext_value(a.w, e >> 24);
}
// four non-negative finite doubles below 2^128; the k-th 16-bit field of a
// SplitMix64 hash of `key` is element k's variate
__device__ __forceinline__ void ext_encode4(const double d[4], unsigned int key, float4 &hi4, unsigned int &ext) {
    unsigned long long h = (unsigned long long)key * 0x9E3779B97F4A7C15ULL;
    h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ULL;
    h = (h ^ (h >> 27)) * 0x94D049BB133111EBULL;
    h ^= h >> 31;
    unsigned int o[4];
    ext = 0u;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(d[k]);
        const long long E = (long long)(b >> 52) - 896;  // the float exponent field
        // exponent and 31 mantissa bits, plus one unit with probability (21 low bits) / 2^21
        unsigned long long c = ((unsigned long long)E << 31) | ((b >> 21) & 0x7fffffffull);
        const unsigned int u = (unsigned int)((h >> (16 * k)) & 0xffffu) << 5;
        c += (u < (unsigned int)(b & 0x1fffffull)) ? 1ull : 0ull;
        o[k] = E > 0 ? (unsigned int)(c >> 8) : 0u;
        ext |= (E > 0 ? (unsigned int)(c & 0xffull) : 0u) << (8 * k);
    }
    hi4 = make_float4(__uint_as_float(o[0]), __uint_as_float(o[1]), __uint_as_float(o[2]), __uint_as_float(o[3]));
}

// A wide buffer b (precision form, batched pass) holds every pattern in FP64
// and occupies the slots of buffers b and b + 1.
__device__ __forceinline__ double *cla_ptr_wide(const View &v, int b, int p, int RS) {
    return reinterpret_cast<double *>(v.partials + (long long)b * v.cla_bytes) + (long long)p * RS;
}

// rescale tables (tree.cpp:163-172), filled from the host with the same libm
// (defined here: the engine is a single CUDA translation unit)
__constant__ double c_thresh[kRescaleTableLen];
__constant__ double c_mult[kRescaleTableLen];
__constant__ int c_incr[kRescaleTableLen];
__constant__ double c_rescale_below, c_reduce_below, c_bail_below;

// Strict IEEE arithmetic: GARLI's CPU build evaluates these expressions without
// fused multiply-add, so the plain form spells every operation out.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

template <typename ST>
__device__ __forceinline__ void load4(const ST *p, double v[4]);
template <>
__device__ __forceinline__ void load4<double>(const double *p, double v[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
template <>
__device__ __forceinline__ void load4<float>(const float *p, double v[4]) {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
template <typename ST>
__device__ __forceinline__ void store4(ST *p, const double v[4]);
template <>
__device__ __forceinline__ void store4<double>(double *p, const double v[4]) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
template <>
__device__ __forceinline__ void store4<float>(float *p, const double v[4]) {
    reinterpret_cast<float4 *>(p)[0] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}

// lanes per pattern for R rate categories (a power of two dividing 32)
template <int R>
struct Lanes {
    static constexpr int G = R <= 1 ? 1 : R <= 2 ? 2 : R <= 4 ? 4 : 8;
};

}  // namespace gb
