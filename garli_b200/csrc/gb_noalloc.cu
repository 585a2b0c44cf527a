// gb_noalloc.cu -- an edge log-likelihood entry point that allocates no device memory.
//
// gb_edge_loglik_static evaluates lnL (and d1, d2) across one branch for
// 4-state data held in caller-owned device arrays, with the same per-site
// arithmetic as the plain FP64 form's edge kernel (k_edge4 with GARLI's
// e-based integer scalers).  It exists for callers that cannot call
// cudaMalloc: code inside a host application that owns every device
// allocation through its own pool (a plugin loaded into such a host), where an
// allocation would bypass the host's accounting or fail once the pool has
// reserved the memory, and code on a latency-critical thread, where
// cudaMalloc's implicit device synchronisation is not allowed.  The kernel's
// only scratch -- one (lnL, d1, d2) partial sum per block -- lives in a
// file-scope __device__ array instead of instance memory.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/garli_b200.h"

// gb_engine.cu: records the message returned by gb_last_error()
void gb_internal_set_last_error(const std::string &msg);

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaPatternsPerBlock = 1024;  // each thread sums 4 patterns of its block's range
constexpr int kNaMaxBlocks = GB_STATIC_EDGE_MAX_PATTERNS / kNaPatternsPerBlock;
constexpr int kNaMaxDevices = 64;
static_assert(GB_STATIC_EDGE_MAX_PATTERNS % kNaPatternsPerBlock == 0, "pattern limit must fill whole blocks");

// Per-block partial sums (lnL, d1, d2) of one call: 3 x 4096 doubles = 96 KiB,
// held by every GPU that loads the library until the process exits.  Calls
// share it: two calls whose kernels overlap on the GPU (different streams, no
// ordering between them) race on it.  Each call writes every slot it later
// reads, so nothing has to be cleared between calls.
static __device__ __align__(256) double g_edge_scratch[3 * kNaMaxBlocks];

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// ((a*b + c*d) + e*f) + g*h, the summation order of GARLI's general rate loops
__device__ __forceinline__ double dot4_seq(const double *p, const double c[4]) {
    return add(add(add(mul(p[0], c[0]), mul(p[1], c[1])), mul(p[2], c[2])), mul(p[3], c[3]));
}

struct EdgeArgs {
    const double *partial;
    const int *partial_scalers;
    const double *child;         // null: the child is a tip given by child_tips
    const int *child_scalers;
    const unsigned char *child_tips;
    const double *mats;          // [P | dP | d2P], each [cat][from][to]
    const double *freqs;
    const double *cat_weights;
    const int *counts;
    const int *const_states;     // 4-bit state mask of a constant pattern, -1 otherwise
    double pinv;
    int has_pinv;
    int npat;
};

// lnL, d1, d2 of pattern p across the branch: GetScorePartial*RateHet
// (tree.cpp:6040, :6172) and GetDerivsPartial* (optimization.cpp:2412, :3063)
template <int R, bool DERIV>
__device__ __forceinline__ void site(const EdgeArgs &a, const double (*M)[R * 16], const double *f,
                                     const double *rp, int p, double &accL, double &acc1, double &acc2) {
    double L[4] = {0, 0, 0, 0}, D1[4] = {0, 0, 0, 0}, D2[4] = {0, 0, 0, 0};
    const bool tip = a.child == nullptr;
    const int m1 = a.partial_scalers[p];
    const int m2 = tip ? 0 : a.child_scalers[p];
    const double *pc = a.partial + (long long)p * R * 4;
    if (!tip) {
        const double *cc = a.child + (long long)p * R * 4;
#pragma unroll
        for (int r = 0; r < R; r++) {
            double part[4], c[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                part[i] = __ldg(pc + r * 4 + i);
                c[i] = __ldg(cc + r * 4 + i);
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                L[i] = add(L[i], mul(mul(dot4_seq(&M[0][16 * r + 4 * i], c), part[i]), rp[r]));
                if (DERIV) {
                    D1[i] = add(D1[i], mul(mul(dot4_seq(&M[1][16 * r + 4 * i], c), part[i]), rp[r]));
                    D2[i] = add(D2[i], mul(mul(dot4_seq(&M[2][16 * r + 4 * i], c), part[i]), rp[r]));
                }
            }
        }
    } else {
        const int code = a.child_tips[p] & 15;
        if (code == 15 || code == 0) {
            // total ambiguity: the partial weighted by the category probabilities
#pragma unroll
            for (int r = 0; r < R; r++)
#pragma unroll
                for (int i = 0; i < 4; i++) L[i] = add(L[i], mul(__ldg(pc + r * 4 + i), rp[r]));
        } else {
            // one state, or a partial ambiguity: states outer, categories inner
            for (int s = 0; s < 4; s++) {
                if (!(code & (1 << s))) continue;
#pragma unroll
                for (int r = 0; r < R; r++) {
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const double part = __ldg(pc + r * 4 + i);
                        L[i] = add(L[i], mul(mul(M[0][16 * r + 4 * i + s], part), rp[r]));
                        if (DERIV) {
                            D1[i] = add(D1[i], mul(mul(M[1][16 * r + 4 * i + s], part), rp[r]));
                            D2[i] = add(D2[i], mul(mul(M[2][16 * r + 4 * i + s], part), rp[r]));
                        }
                    }
                }
            }
        }
    }
    double siteL = add(add(add(mul(L[0], f[0]), mul(L[1], f[1])), mul(L[2], f[2])), mul(L[3], f[3]));
    const int cb = a.has_pinv ? a.const_states[p] : -1;
    if (cb >= 0) {
        double btot = 0.0;
        for (int s = 0; s < 4; s++)
            if (cb & (1 << s)) btot = add(btot, f[s]);
        if (DERIV) {
            const double e = tip ? exp((double)m1) : exp(add((double)m2, (double)m1));
            siteL = add(siteL, mul(mul(a.pinv, btot), e));
        } else if (m1 + m2 == 0) {
            siteL = add(siteL, mul(a.pinv, btot));
        } else {
            siteL = add(siteL, mul(mul(a.pinv, btot), exp(add((double)m1, (double)m2))));
        }
    }
    const double lg = log(siteL);
    const double u = (DERIV && !tip) ? sub(sub(lg, (double)m2), (double)m1) : sub(sub(lg, (double)m1), (double)m2);
    const double cnt = (double)a.counts[p];
    accL = add(accL, mul(cnt, u));
    if (DERIV) {
        const double sd1 = add(add(add(mul(D1[0], f[0]), mul(D1[1], f[1])), mul(D1[2], f[2])), mul(D1[3], f[3])) / siteL;
        const double sd2 =
            sub(add(add(add(mul(D2[0], f[0]), mul(D2[1], f[1])), mul(D2[2], f[2])), mul(D2[3], f[3])) / siteL,
                mul(sd1, sd1));
        acc1 = add(acc1, mul(cnt, sd1));
        acc2 = add(acc2, mul(cnt, sd2));
    }
}

// One block per kNaPatternsPerBlock patterns; block b writes scratch[3b .. 3b+2].
template <int R, bool DERIV>
__global__ void __launch_bounds__(kNaThreads) k_edge4_static(EdgeArgs a, double *scratch) {
    __shared__ double M[3][R * 16];
    __shared__ double f[4], rp[R];
    __shared__ double red[3][kNaThreads / 32];
    for (int i = threadIdx.x; i < R * 16; i += blockDim.x) {
        M[0][i] = a.mats[i];
        M[1][i] = DERIV ? a.mats[R * 16 + i] : 0.0;
        M[2][i] = DERIV ? a.mats[2 * R * 16 + i] : 0.0;
    }
    if (threadIdx.x < 4) f[threadIdx.x] = a.freqs[threadIdx.x];
    if (threadIdx.x < R) rp[threadIdx.x] = a.cat_weights[threadIdx.x];
    __syncthreads();
    double accL = 0.0, acc1 = 0.0, acc2 = 0.0;
    const int p0 = blockIdx.x * kNaPatternsPerBlock;
    const int p1 = min(a.npat, p0 + kNaPatternsPerBlock);
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) site<R, DERIV>(a, M, f, rp, p, accL, acc1, acc2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        accL += __shfl_down_sync(0xffffffffu, accL, o);
        acc1 += __shfl_down_sync(0xffffffffu, acc1, o);
        acc2 += __shfl_down_sync(0xffffffffu, acc2, o);
    }
    const int w = threadIdx.x / 32;
    if (threadIdx.x % 32 == 0) {
        red[0][w] = accL;
        red[1][w] = acc1;
        red[2][w] = acc2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int i = 0; i < kNaThreads / 32; i++) {
            s0 += red[0][i];
            s1 += red[1][i];
            s2 += red[2][i];
        }
        scratch[3 * blockIdx.x] = s0;
        scratch[3 * blockIdx.x + 1] = s1;
        scratch[3 * blockIdx.x + 2] = s2;
    }
}

// Fixed-order sum of the nblocks partial sums into out[0..2] (one block).
__global__ void __launch_bounds__(kNaThreads) k_reduce3_static(const double *scratch, int nblocks, double *out) {
    __shared__ double s[3][kNaThreads];
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a += scratch[3 * i];
        b += scratch[3 * i + 1];
        c += scratch[3 * i + 2];
    }
    s[0][threadIdx.x] = a;
    s[1][threadIdx.x] = b;
    s[2][threadIdx.x] = c;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s[0][threadIdx.x] += s[0][threadIdx.x + w];
            s[1][threadIdx.x] += s[1][threadIdx.x + w];
            s[2][threadIdx.x] += s[2][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s[0][0];
        out[1] = s[1][0];
        out[2] = s[2][0];
    }
}

// Each launch's own result: cudaLaunchKernel returns the error of this launch,
// so an unrelated error left pending earlier on the thread is neither reported
// as this call's nor cleared for its owner.
template <bool D>
cudaError_t launch_edge(int R, int nblocks, cudaStream_t st, const EdgeArgs &a, double *scratch) {
    void *f = nullptr;
    switch (R) {
        case 1: f = (void *)k_edge4_static<1, D>; break;
        case 2: f = (void *)k_edge4_static<2, D>; break;
        case 3: f = (void *)k_edge4_static<3, D>; break;
        case 4: f = (void *)k_edge4_static<4, D>; break;
        case 5: f = (void *)k_edge4_static<5, D>; break;
        case 6: f = (void *)k_edge4_static<6, D>; break;
        case 7: f = (void *)k_edge4_static<7, D>; break;
        default: f = (void *)k_edge4_static<8, D>; break;
    }
    EdgeArgs args = a;
    void *kargs[] = {&args, &scratch};
    return cudaLaunchKernel(f, dim3(nblocks), dim3(kNaThreads), kargs, 0, st);
}

// Device address of g_edge_scratch, looked up once per device with that
// device current and kept for the life of the process: a cudaDeviceReset on
// that device invalidates it, and the entry point must not be called after one.  In host code the name g_edge_scratch is only a host-side
// stand-in for the symbol; handing it to a kernel would fault or, where the
// GPU can reach host memory, silently use the wrong memory.
std::mutex g_scratch_mu;
double *g_scratch_ptr[kNaMaxDevices] = {};

int scratch_address(int device, double **out) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_edge_scratch);
        if (e != cudaSuccess || !p) {
            gb_internal_set_last_error(std::string("gb_edge_loglik_static: cudaGetSymbolAddress: ") +
                                       cudaGetErrorString(e));
            return GB_ERROR_GENERAL;
        }
        g_scratch_ptr[device] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[device];
    return GB_SUCCESS;
}

int fail(int code, const char *msg) {
    gb_internal_set_last_error(std::string("gb_edge_loglik_static: ") + msg);
    return code;
}

}  // namespace

extern "C" int gb_edge_loglik_static(int resourceNumber, int categoryCount, int patternCount, const double *partial,
                                     const int *partialScalers, const double *child, const int *childScalers,
                                     const unsigned char *childTipCodes, const double *matrices,
                                     const double *stateFrequencies, const double *categoryWeights,
                                     const int *patternCounts, const int *constantStates, double pinv, int hasPinv,
                                     int derivatives, void *stream, double *out) {
    if (categoryCount < 1 || categoryCount > 8) return fail(GB_ERROR_OUT_OF_RANGE, "categoryCount must be 1..8");
    if (patternCount < 1 || patternCount > GB_STATIC_EDGE_MAX_PATTERNS)
        return fail(GB_ERROR_OUT_OF_RANGE,
                    "patternCount must be 1..GB_STATIC_EDGE_MAX_PATTERNS (4194304): the scratch array is fixed");
    if (!partial || !partialScalers || !matrices || !stateFrequencies || !categoryWeights || !patternCounts || !out)
        return fail(GB_ERROR_OUT_OF_RANGE, "null input or output pointer");
    if ((child == nullptr) == (childTipCodes == nullptr))
        return fail(GB_ERROR_OUT_OF_RANGE, "give exactly one of child (a CLA) and childTipCodes (a tip)");
    if (child && !childScalers) return fail(GB_ERROR_OUT_OF_RANGE, "a CLA child needs childScalers");
    if (hasPinv && !constantStates) return fail(GB_ERROR_OUT_OF_RANGE, "hasPinv needs constantStates");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(GB_ERROR_NO_DEVICE, "no CUDA device");
    if (resourceNumber < 0 || resourceNumber >= ndev || resourceNumber >= kNaMaxDevices)
        return fail(GB_ERROR_OUT_OF_RANGE, "resourceNumber is not a device ordinal");
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(resourceNumber) != cudaSuccess) return fail(GB_ERROR_NO_DEVICE, "cudaSetDevice failed");
    double *scratch = nullptr;
    int rc = scratch_address(resourceNumber, &scratch);
    if (rc == GB_SUCCESS) {
        EdgeArgs a;
        a.partial = partial;
        a.partial_scalers = partialScalers;
        a.child = child;
        a.child_scalers = childScalers;
        a.child_tips = childTipCodes;
        a.mats = matrices;
        a.freqs = stateFrequencies;
        a.cat_weights = categoryWeights;
        a.counts = patternCounts;
        a.const_states = constantStates;
        a.pinv = pinv;
        a.has_pinv = hasPinv ? 1 : 0;
        a.npat = patternCount;
        const int nblocks = (patternCount + kNaPatternsPerBlock - 1) / kNaPatternsPerBlock;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        cudaError_t e = derivatives ? launch_edge<true>(categoryCount, nblocks, st, a, scratch)
                                    : launch_edge<false>(categoryCount, nblocks, st, a, scratch);
        if (e == cudaSuccess) {
            const double *sc = scratch;
            int nb = nblocks;
            void *rargs[] = {(void *)&sc, &nb, &out};
            e = cudaLaunchKernel((void *)k_reduce3_static, dim3(1), dim3(kNaThreads), rargs, 0, st);
        }
        if (e != cudaSuccess) rc = fail(GB_ERROR_GENERAL, cudaGetErrorString(e));
    }
    cudaSetDevice(prev);
    return rc;
}
