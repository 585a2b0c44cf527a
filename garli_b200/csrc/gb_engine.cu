// gb_engine.cu -- instance management and the C ABI of the garli_b200 engine.
//
// One instance = one GARLI data subset on one GPU (the role of a beagle
// instance created by SubsetCalculationManager, subsetcalculationmanager.cpp:105).
// All device memory is allocated at creation; every call after that only
// launches kernels on the instance's stream and, for calls that return
// results, copies a few bytes back.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/garli_b200.h"
#include "gb_common.cuh"
#include "gb_dna.cuh"
#include "gb_nstate.cuh"
#include "gb_pmat.cuh"

namespace gb {

static thread_local std::string g_last_error;

struct Instance {
    int device = 0;
    int ntip = 0, nbuf = 0, S = 0, R = 0, npat = 0, npat_pad = 0, neigen = 0, nmat = 0;
    long flags = 0;
    bool mixed = false;
    size_t elem = 8;
    cudaStream_t stream = nullptr;
    // device memory
    void *d_partials = nullptr;
    int *d_scalers = nullptr;
    uint8_t *d_tips = nullptr;
    int *d_counts = nullptr, *d_const = nullptr;
    double *d_mats = nullptr, *d_eigen = nullptr;
    double *d_freqs = nullptr, *d_rates = nullptr, *d_rprobs = nullptr;
    int *d_status = nullptr;
    double *d_block_sums = nullptr, *d_result = nullptr, *d_site_lnl = nullptr;
    // pinned result staging
    double *h_result = nullptr;
    int *h_status = nullptr;
    // host state
    std::vector<double> h_rates;
    double pinv = 0.0;
    int has_pinv = 0, last_const = -1;
    std::vector<int> rank;  // per CLA buffer (condlike.h rescaleRank)
    long long launches = 0;
    long long bytes = 0;
    bool site_valid = false;
    // optional CLA kernel timing (CUDA events on the instance stream)
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    std::vector<long long> ev_updates;
    double cla_ms = 0.0;
    long long cla_launches_timed = 0, cla_updates_timed = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_edge;
    double edge_ms = 0.0;
    long long edge_timed = 0;

    long long cla_stride() const { return (long long)npat_pad * R * S; }
    long long mat_stride() const { return 3LL * R * S * S; }
    long long eig_stride() const { return (long long)S + 2LL * S * S; }
};

static std::mutex g_mu;
static std::vector<Instance *> g_inst;

static Instance *get(int h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h < 0 || h >= (int)g_inst.size()) return nullptr;
    return g_inst[h];
}

#define GB_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);             \
            return e_ == cudaErrorMemoryAllocation ? GB_ERROR_OUT_OF_MEMORY : GB_ERROR_GENERAL; \
        }                                                                                  \
    } while (0)

static int check_launch(Instance *I) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_error = std::string("kernel launch: ") + cudaGetErrorString(e);
        return GB_ERROR_GENERAL;
    }
    I->launches++;
    return GB_SUCCESS;
}

static View make_view(Instance *I) {
    View v;
    v.partials = I->d_partials;
    v.scalers = I->d_scalers;
    v.tips = I->d_tips;
    v.mats = I->d_mats;
    v.counts = I->d_counts;
    v.const_states = I->d_const;
    v.freqs = I->d_freqs;
    v.rate_probs = I->d_rprobs;
    v.status = I->d_status;
    v.block_sums = I->d_block_sums;
    v.site_lnl = I->d_site_lnl;
    v.cla_stride = I->cla_stride();
    v.mat_stride = I->mat_stride();
    v.npat = I->npat;
    v.npat_pad = I->npat_pad;
    v.ntip = I->ntip;
    v.last_const = I->last_const;
    v.has_pinv = I->has_pinv;
    v.rescale_every = 16;
    v.pinv = I->pinv;
    return v;
}

// rescale tables with the host libm, exactly as Tree::SetTreeStatics (tree.cpp:163-172)
static int upload_rescale_tables() {
    double thresh[kRescaleTableLen], mult[kRescaleTableLen];
    int incr[kRescaleTableLen];
    const double rescaleBelow = std::exp(-24.0);
    const double reduceBelow = 1.0e-190, bailBelow = 1.0e-250;
    const double maxMult = 1.0 / bailBelow;
    for (int i = 0; i < kRescaleTableLen; i++) {
        incr[i] = i * 7 - (int)std::log(rescaleBelow);
        thresh[i] = std::exp((double)(-incr[i]));
        mult[i] = std::min(std::exp((double)incr[i]), maxMult);
    }
    GB_CUDA(cudaMemcpyToSymbol(c_thresh, thresh, sizeof(thresh)));
    GB_CUDA(cudaMemcpyToSymbol(c_mult, mult, sizeof(mult)));
    GB_CUDA(cudaMemcpyToSymbol(c_incr, incr, sizeof(incr)));
    GB_CUDA(cudaMemcpyToSymbol(c_rescale_below, &rescaleBelow, sizeof(double)));
    GB_CUDA(cudaMemcpyToSymbol(c_reduce_below, &reduceBelow, sizeof(double)));
    GB_CUDA(cudaMemcpyToSymbol(c_bail_below, &bailBelow, sizeof(double)));
    return GB_SUCCESS;
}

// ---------------------------------------------------------------------------
// kernel dispatch
// ---------------------------------------------------------------------------
template <typename ST, bool G>
static void launch_cla4(int R, dim3 grid, cudaStream_t st, const View &v, const LevelOps &ops) {
    switch (R) {
        case 1: k_cla4<ST, 1, G><<<grid, kThreads, 0, st>>>(v, ops); break;
        case 2: k_cla4<ST, 2, G><<<grid, kThreads, 0, st>>>(v, ops); break;
        case 3: k_cla4<ST, 3, G><<<grid, kThreads, 0, st>>>(v, ops); break;
        case 4: k_cla4<ST, 4, G><<<grid, kThreads, 0, st>>>(v, ops); break;
        case 5: k_cla4<ST, 5, G><<<grid, kThreads, 0, st>>>(v, ops); break;
        case 6: k_cla4<ST, 6, G><<<grid, kThreads, 0, st>>>(v, ops); break;
        case 7: k_cla4<ST, 7, G><<<grid, kThreads, 0, st>>>(v, ops); break;
        default: k_cla4<ST, 8, G><<<grid, kThreads, 0, st>>>(v, ops); break;
    }
}

template <typename ST, bool G, bool D>
static void launch_edge4(int R, int grid, cudaStream_t st, const View &v, int pb, int cb, int mat, int tip,
                         int ws) {
    switch (R) {
        case 1: k_edge4<ST, 1, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 2: k_edge4<ST, 2, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 3: k_edge4<ST, 3, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 4: k_edge4<ST, 4, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 5: k_edge4<ST, 5, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 6: k_edge4<ST, 6, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 7: k_edge4<ST, 7, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        default: k_edge4<ST, 8, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
    }
}

static int ns_cla_tile(const Instance *I, size_t *smem) {
    const int RS = I->R * I->S, RSS = RS * I->S;
    int tp = 64;
    while (tp > 1 && (size_t)(2 * RSS + 3 * tp * RS + tp) * 8 > 160 * 1024) tp >>= 1;
    *smem = (size_t)(2 * RSS + 3 * tp * RS + tp) * 8;
    return tp;
}
static int ns_edge_tile(const Instance *I, size_t *smem) {
    const int RS = I->R * I->S, RSS = RS * I->S;
    int tp = 64;
    while (tp > 1 && (size_t)(3 * RSS + 5 * tp * RS + I->S + I->R) * 8 > 180 * 1024) tp >>= 1;
    *smem = (size_t)(3 * RSS + 5 * tp * RS + I->S + I->R) * 8;
    return tp;
}

static int set_smem_attrs() {
    const int big = 200 * 1024;
    GB_CUDA(cudaFuncSetAttribute(k_cla_ns<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    GB_CUDA(cudaFuncSetAttribute(k_cla_ns<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    GB_CUDA(cudaFuncSetAttribute(k_edge_ns<double, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    GB_CUDA(cudaFuncSetAttribute(k_edge_ns<double, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    GB_CUDA(cudaFuncSetAttribute(k_edge_ns<float, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    GB_CUDA(cudaFuncSetAttribute(k_edge_ns<float, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    GB_CUDA(cudaFuncSetAttribute(k_pmats, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    return GB_SUCCESS;
}

static int launch_level(Instance *I, const std::vector<DevOp> &ops, int rescaleEvery) {
    View v = make_view(I);
    v.rescale_every = rescaleEvery;
    for (size_t b = 0; b < ops.size(); b += kMaxLevelOps) {
        LevelOps L;
        L.n = (int)std::min<size_t>(kMaxLevelOps, ops.size() - b);
        for (int i = 0; i < L.n; i++) L.op[i] = ops[b + i];
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (I->timing) {
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, I->stream);
        }
        if (I->S == 4) {
            const int G = I->R <= 1 ? 1 : I->R <= 2 ? 2 : I->R <= 4 ? 4 : 8;
            const int ppb = kThreads / G;
            dim3 grid((I->npat + ppb - 1) / ppb, L.n);
            if (I->mixed) launch_cla4<float, false>(I->R, grid, I->stream, v, L);
            else launch_cla4<double, true>(I->R, grid, I->stream, v, L);
        } else {
            size_t smem;
            const int tp = ns_cla_tile(I, &smem);
            dim3 grid((I->npat + tp - 1) / tp, L.n);
            if (I->mixed) k_cla_ns<float, false><<<grid, kThreads, smem, I->stream>>>(v, L, I->S, I->R, tp);
            else k_cla_ns<double, true><<<grid, kThreads, smem, I->stream>>>(v, L, I->S, I->R, tp);
        }
        int rc = check_launch(I);
        if (rc) return rc;
        if (I->timing) {
            cudaEventRecord(e1, I->stream);
            I->ev.emplace_back(e0, e1);
            I->ev_updates.push_back((long long)L.n * I->npat);
        }
    }
    return GB_SUCCESS;
}

static void resolve_timing(Instance *I) {
    if (I->ev.empty() && I->ev_edge.empty()) return;
    cudaStreamSynchronize(I->stream);
    for (size_t i = 0; i < I->ev.size(); i++) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, I->ev[i].first, I->ev[i].second);
        I->cla_ms += ms;
        I->cla_launches_timed++;
        I->cla_updates_timed += I->ev_updates[i];
        cudaEventDestroy(I->ev[i].first);
        cudaEventDestroy(I->ev[i].second);
    }
    for (auto &pr : I->ev_edge) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pr.first, pr.second);
        I->edge_ms += ms;
        I->edge_timed++;
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    I->ev.clear();
    I->ev_updates.clear();
    I->ev_edge.clear();
}

}  // namespace gb

using namespace gb;

extern "C" {

const char *gb_last_error(void) { return g_last_error.c_str(); }

int gb_get_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int gb_create_instance(int tipCount, int partialsBufferCount, int stateCount, int patternCount,
                       int eigenBufferCount, int matrixBufferCount, int categoryCount, int resourceNumber,
                       long flags, gb_instance_details *details) {
    if (tipCount < 2 || partialsBufferCount < 1 || patternCount < 1 || eigenBufferCount < 1 ||
        matrixBufferCount < 1 || categoryCount < 1 || categoryCount > 8)
        return GB_ERROR_OUT_OF_RANGE;
    if (stateCount != 4 && stateCount != 20 && stateCount != 61) return GB_ERROR_NO_IMPLEMENTATION;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_last_error = "no CUDA device";
        return GB_ERROR_NO_DEVICE;
    }
    if (resourceNumber < 0 || resourceNumber >= ndev) return GB_ERROR_NO_RESOURCE;
    auto *I = new Instance();
    I->device = resourceNumber;
    I->ntip = tipCount;
    I->nbuf = partialsBufferCount;
    I->S = stateCount;
    I->R = categoryCount;
    I->npat = patternCount;
    I->npat_pad = (patternCount + 127) / 128 * 128;
    I->neigen = eigenBufferCount;
    I->nmat = matrixBufferCount;
    I->mixed = (flags & GB_FLAG_MIXED_FP32) != 0;
    I->flags = I->mixed ? GB_FLAG_MIXED_FP32 : GB_FLAG_PLAIN_FP64;
    I->elem = I->mixed ? 4 : 8;
    I->rank.assign(partialsBufferCount, 0);
    I->h_rates.assign(categoryCount, 1.0);
    auto fail = [&](int rc) {
        if (I->stream) cudaStreamDestroy(I->stream);
        delete I;
        return rc;
    };
    if (cudaSetDevice(resourceNumber) != cudaSuccess) return fail(GB_ERROR_NO_RESOURCE);
    int rc = upload_rescale_tables();
    if (rc) return fail(rc);
    rc = set_smem_attrs();
    if (rc) return fail(rc);
    if (cudaStreamCreateWithFlags(&I->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(GB_ERROR_GENERAL);
    const size_t P = I->npat_pad;
    const size_t cla_bytes = (size_t)I->nbuf * P * I->R * I->S * I->elem;
    struct A {
        void **p;
        size_t n;
    } allocs[] = {
        {&I->d_partials, cla_bytes},
        {(void **)&I->d_scalers, (size_t)I->nbuf * P * sizeof(int)},
        {(void **)&I->d_tips, (size_t)I->ntip * P},
        {(void **)&I->d_counts, P * sizeof(int)},
        {(void **)&I->d_const, P * sizeof(int)},
        {(void **)&I->d_mats, (size_t)I->nmat * I->mat_stride() * sizeof(double)},
        {(void **)&I->d_eigen, (size_t)I->neigen * I->eig_stride() * sizeof(double)},
        {(void **)&I->d_freqs, (size_t)I->S * sizeof(double)},
        {(void **)&I->d_rates, (size_t)I->R * sizeof(double)},
        {(void **)&I->d_rprobs, (size_t)I->R * sizeof(double)},
        {(void **)&I->d_status, sizeof(int)},
        {(void **)&I->d_block_sums, (size_t)kMaxScoreBlocks * 3 * sizeof(double)},
        {(void **)&I->d_result, 4 * sizeof(double)},
        {(void **)&I->d_site_lnl, P * sizeof(double)},
    };
    for (auto &a : allocs) {
        if (cudaMalloc(a.p, a.n) != cudaSuccess) {
            g_last_error = "cudaMalloc failed";
            for (auto &b : allocs)
                if (*b.p) cudaFree(*b.p);
            cudaStreamDestroy(I->stream);
            delete I;
            return GB_ERROR_OUT_OF_MEMORY;
        }
        I->bytes += (long long)a.n;
        cudaMemsetAsync(*a.p, 0, a.n, I->stream);
    }
    if (cudaMallocHost((void **)&I->h_result, 4 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost((void **)&I->h_status, sizeof(int)) != cudaSuccess) {
        for (auto &b : allocs) cudaFree(*b.p);
        delete I;
        return GB_ERROR_OUT_OF_MEMORY;
    }
    // default tips: missing everywhere; default weights 1 (padding stays 0)
    std::vector<int> ones(P, 0);
    for (int i = 0; i < patternCount; i++) ones[i] = 1;
    cudaMemcpyAsync(I->d_counts, ones.data(), P * sizeof(int), cudaMemcpyHostToDevice, I->stream);
    cudaMemsetAsync(I->d_tips, stateCount == 4 ? 15 : stateCount, (size_t)I->ntip * P, I->stream);
    std::vector<double> one(I->R, 1.0), pr(I->R, 1.0 / I->R), fr(I->S, 1.0 / I->S);
    cudaMemcpyAsync(I->d_rates, one.data(), I->R * sizeof(double), cudaMemcpyHostToDevice, I->stream);
    cudaMemcpyAsync(I->d_rprobs, pr.data(), I->R * sizeof(double), cudaMemcpyHostToDevice, I->stream);
    cudaMemcpyAsync(I->d_freqs, fr.data(), I->S * sizeof(double), cudaMemcpyHostToDevice, I->stream);
    if (cudaStreamSynchronize(I->stream) != cudaSuccess) {
        g_last_error = "instance initialisation failed";
        return GB_ERROR_GENERAL;
    }
    int h;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_inst.push_back(I);
        h = (int)g_inst.size() - 1;
    }
    if (details) {
        details->resourceNumber = resourceNumber;
        details->flags = I->flags;
        details->paddedPatterns = I->npat_pad;
        details->deviceBytes = I->bytes;
        cudaDeviceProp prop;
        cudaGetDeviceProperties(&prop, resourceNumber);
        std::snprintf(details->deviceName, sizeof(details->deviceName), "%s", prop.name);
    }
    return h;
}

int gb_finalize_instance(int instance) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    cudaStreamSynchronize(I->stream);
    resolve_timing(I);
    void *ptrs[] = {I->d_partials, I->d_scalers, I->d_tips, I->d_counts, I->d_const, I->d_mats,
                    I->d_eigen, I->d_freqs, I->d_rates, I->d_rprobs, I->d_status, I->d_block_sums,
                    I->d_result, I->d_site_lnl};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    cudaFreeHost(I->h_result);
    cudaFreeHost(I->h_status);
    cudaStreamDestroy(I->stream);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_inst[instance] = nullptr;
    }
    delete I;
    return GB_SUCCESS;
}

int gb_set_tip_states(int instance, int tipIndex, const unsigned char *codes) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (tipIndex < 0 || tipIndex >= I->ntip || !codes) return GB_ERROR_OUT_OF_RANGE;
    const int miss = I->S == 4 ? 15 : I->S;
    for (int p = 0; p < I->npat; p++)
        if (I->S == 4 ? (codes[p] & ~15) != 0 : codes[p] > miss) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(I->d_tips + (size_t)tipIndex * I->npat_pad, codes, I->npat, cudaMemcpyHostToDevice,
                            I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_set_pattern_weights(int instance, const int *counts) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(I->d_counts, counts, I->npat * sizeof(int), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_set_constant_patterns(int instance, int lastConst, const int *constStates) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (lastConst >= I->npat || lastConst < -1) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    I->last_const = lastConst;
    if (lastConst >= 0) {
        for (int p = 0; p <= lastConst; p++)
            if (constStates[p] < 0 || constStates[p] > (I->S == 4 ? 15 : I->S - 1)) return GB_ERROR_OUT_OF_RANGE;
        GB_CUDA(cudaMemcpyAsync(I->d_const, constStates, (lastConst + 1) * sizeof(int), cudaMemcpyHostToDevice,
                                I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
    }
    return GB_SUCCESS;
}

int gb_set_state_frequencies(int instance, const double *freqs) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(I->d_freqs, freqs, I->S * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_set_category_rates(int instance, const double *rates) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    I->h_rates.assign(rates, rates + I->R);
    GB_CUDA(cudaMemcpyAsync(I->d_rates, rates, I->R * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_set_category_weights(int instance, const double *weights) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(I->d_rprobs, weights, I->R * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_set_invariant_sites(int instance, double pinv, int hasPinv) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!(pinv >= 0.0 && pinv < 1.0)) return GB_ERROR_OUT_OF_RANGE;
    I->pinv = pinv;
    I->has_pinv = hasPinv ? 1 : 0;
    return GB_SUCCESS;
}

int gb_set_eigen_decomposition(int instance, int eigenIndex, const double *U, const double *Uinv,
                               const double *lambda) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (eigenIndex < 0 || eigenIndex >= I->neigen) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    const int S = I->S;
    std::vector<double> buf(I->eig_stride());
    std::memcpy(buf.data(), lambda, S * sizeof(double));
    std::memcpy(buf.data() + S, U, (size_t)S * S * sizeof(double));
    std::memcpy(buf.data() + S + S * S, Uinv, (size_t)S * S * sizeof(double));
    GB_CUDA(cudaMemcpyAsync(I->d_eigen + (size_t)eigenIndex * I->eig_stride(), buf.data(),
                            buf.size() * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_update_transition_matrices(int instance, const gb_transmat_operation *ops, int count) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (count < 0) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    for (int b = 0; b < count; b += kMaxTransOps) {
        TransOps T;
        T.n = std::min(kMaxTransOps, count - b);
        for (int i = 0; i < T.n; i++) {
            const gb_transmat_operation &o = ops[b + i];
            if (o.destTransMatIndex < 0 || o.destTransMatIndex >= I->nmat || o.eigenIndex < 0 ||
                o.eigenIndex >= I->neigen || !(o.edgeLength >= 0.0))
                return GB_ERROR_OUT_OF_RANGE;
            T.op[i].dest = o.destTransMatIndex;
            T.op[i].eigen = o.eigenIndex;
            T.op[i].derivs = o.calcDerivs;
            T.op[i].t = o.edgeLength;
        }
        const size_t smem = 3 * (size_t)I->R * I->S * sizeof(double);
        k_pmats<<<T.n, kThreads, smem, I->stream>>>(I->d_eigen, I->eig_stride(), I->S, I->R, I->d_rates, I->pinv,
                                                     I->has_pinv, T, I->d_mats, I->mat_stride());
        int rc = check_launch(I);
        if (rc) return rc;
    }
    return GB_SUCCESS;
}

int gb_set_transition_matrix(int instance, int matrixIndex, const double *P, const double *D1, const double *D2) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (matrixIndex < 0 || matrixIndex >= I->nmat) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    const size_t n = (size_t)I->R * I->S * I->S;
    double *dst = I->d_mats + (size_t)matrixIndex * I->mat_stride();
    GB_CUDA(cudaMemcpyAsync(dst, P, n * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    if (D1) GB_CUDA(cudaMemcpyAsync(dst + n, D1, n * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    if (D2) GB_CUDA(cudaMemcpyAsync(dst + 2 * n, D2, n * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_update_partials(int instance, const gb_cla_operation *ops, int count, int rescaleEvery) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (count < 0) return GB_ERROR_OUT_OF_RANGE;
    if (count == 0) return GB_SUCCESS;
    cudaSetDevice(I->device);
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return ops[a].opDepLevel < ops[b].opDepLevel; });
    const int nt = I->ntip, nb = I->nbuf;
    auto is_tip = [&](int b) { return b >= 0 && b < nt; };
    auto is_cla = [&](int b) { return b >= nt && b < nt + nb; };
    std::vector<DevOp> level;
    int cur = ops[order[0]].opDepLevel;
    for (int k = 0; k <= count; k++) {
        if (k == count || ops[order[k]].opDepLevel != cur) {
            int rc = launch_level(I, level, rescaleEvery);
            if (rc) return rc;
            level.clear();
            if (k == count) break;
            cur = ops[order[k]].opDepLevel;
        }
        const gb_cla_operation &o = ops[order[k]];
        if (!is_cla(o.destClaIndex) || !(is_tip(o.childClaIndex1) || is_cla(o.childClaIndex1)) ||
            !(is_tip(o.childClaIndex2) || is_cla(o.childClaIndex2)) || o.transMatIndex1 < 0 ||
            o.transMatIndex1 >= I->nmat || o.transMatIndex2 < 0 || o.transMatIndex2 >= I->nmat)
            return GB_ERROR_OUT_OF_RANGE;
        DevOp d;
        int c1 = o.childClaIndex1, c2 = o.childClaIndex2, p1 = o.transMatIndex1, p2 = o.transMatIndex2;
        if (is_tip(c1) && is_cla(c2)) {
            std::swap(c1, c2);
            std::swap(p1, p2);
        }
        const int dest = o.destClaIndex - nt;
        int rank;
        if (is_cla(c1) && is_cla(c2)) {
            d.kind = kIntInt;
            rank = 2 + I->rank[c1 - nt] + I->rank[c2 - nt];
        } else if (is_cla(c1)) {
            d.kind = kIntTip;
            rank = I->rank[c1 - nt] + 2;
        } else {
            d.kind = kTipTip;
            rank = 2;
        }
        d.dest = dest;
        d.c1 = is_cla(c1) ? c1 - nt : c1;
        d.c2 = is_cla(c2) ? c2 - nt : c2;
        d.p1 = p1;
        d.p2 = p2;
        d.rescale = (!I->mixed && rank >= rescaleEvery) ? 1 : 0;
        I->rank[dest] = d.rescale ? 0 : rank;
        level.push_back(d);
    }
    return GB_SUCCESS;
}

static int edge_impl(Instance *I, const gb_scoring_operation *op, double *out, bool sync) {
    const int nt = I->ntip;
    const int pb = op->childClaIndex1 - nt;
    const int cb = op->childClaIndex2;
    if (pb < 0 || pb >= I->nbuf || cb < 0 || cb >= nt + I->nbuf || op->transMatIndex < 0 ||
        op->transMatIndex >= I->nmat)
        return GB_ERROR_OUT_OF_RANGE;
    const int tip = cb < nt;
    const int cidx = tip ? cb : cb - nt;
    View v = make_view(I);
    const bool D = op->derivatives != 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (I->timing) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, I->stream);
    }
    int nblocks;
    if (I->S == 4) {
        nblocks = std::min(kMaxScoreBlocks, (I->npat + kThreads - 1) / kThreads);
        if (I->mixed) {
            if (D) launch_edge4<float, false, true>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
            else launch_edge4<float, false, false>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
        } else {
            if (D) launch_edge4<double, true, true>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
            else launch_edge4<double, true, false>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
        }
    } else {
        size_t smem;
        const int tp = ns_edge_tile(I, &smem);
        nblocks = std::min(kMaxScoreBlocks, (I->npat + tp - 1) / tp);
        if (I->mixed) {
            if (D) k_edge_ns<float, false, true><<<nblocks, kThreads, smem, I->stream>>>(v, pb, cidx, op->transMatIndex, tip, 1, I->S, I->R, tp);
            else k_edge_ns<float, false, false><<<nblocks, kThreads, smem, I->stream>>>(v, pb, cidx, op->transMatIndex, tip, 1, I->S, I->R, tp);
        } else {
            if (D) k_edge_ns<double, true, true><<<nblocks, kThreads, smem, I->stream>>>(v, pb, cidx, op->transMatIndex, tip, 1, I->S, I->R, tp);
            else k_edge_ns<double, true, false><<<nblocks, kThreads, smem, I->stream>>>(v, pb, cidx, op->transMatIndex, tip, 1, I->S, I->R, tp);
        }
    }
    int rc = check_launch(I);
    if (rc) return rc;
    k_reduce3<<<1, kThreads, 0, I->stream>>>(I->d_block_sums, nblocks, I->d_result);
    rc = check_launch(I);
    if (rc) return rc;
    if (I->timing) {
        cudaEventRecord(e1, I->stream);
        I->ev_edge.emplace_back(e0, e1);
    }
    I->site_valid = true;
    if (!sync) return GB_SUCCESS;
    GB_CUDA(cudaMemcpyAsync(I->h_result, I->d_result, 3 * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaMemcpyAsync(I->h_status, I->d_status, sizeof(int), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    out[0] = I->h_result[0];
    out[1] = D ? I->h_result[1] : 0.0;
    out[2] = D ? I->h_result[2] : 0.0;
    if (*I->h_status & kStatusRescaleRetry) {
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        return GB_ERROR_RESCALE_RETRY;
    }
    if (!std::isfinite(out[0])) return GB_ERROR_FLOATING_POINT;
    return GB_SUCCESS;
}

int gb_calculate_edge(int instance, const gb_scoring_operation *op, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!op || !out) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    return edge_impl(I, op, out, true);
}

int gb_get_site_log_likelihoods(int instance, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!I->site_valid) return GB_ERROR_GENERAL;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(out, I->d_site_lnl, I->npat * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_get_partials(int instance, int bufferIndex, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    const int b = bufferIndex - I->ntip;
    if (b < 0 || b >= I->nbuf) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    const size_t n = (size_t)I->npat * I->R * I->S;
    const char *src = (const char *)I->d_partials + (size_t)b * I->cla_stride() * I->elem;
    if (!I->mixed) {
        GB_CUDA(cudaMemcpyAsync(out, src, n * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
    } else {
        std::vector<float> tmp(n);
        GB_CUDA(cudaMemcpyAsync(tmp.data(), src, n * sizeof(float), cudaMemcpyDeviceToHost, I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        for (size_t i = 0; i < n; i++) out[i] = tmp[i];
    }
    return GB_SUCCESS;
}

int gb_get_scale_factors(int instance, int bufferIndex, int *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    const int b = bufferIndex - I->ntip;
    if (b < 0 || b >= I->nbuf) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(out, I->d_scalers + (size_t)b * I->npat_pad, I->npat * sizeof(int),
                            cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_get_transition_matrix(int instance, int matrixIndex, int which, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (matrixIndex < 0 || matrixIndex >= I->nmat || which < 0 || which > 2) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    const size_t n = (size_t)I->R * I->S * I->S;
    GB_CUDA(cudaMemcpyAsync(out, I->d_mats + (size_t)matrixIndex * I->mat_stride() + which * n,
                            n * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_get_rescale_rank(int instance, int bufferIndex) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    const int b = bufferIndex - I->ntip;
    if (b < 0 || b >= I->nbuf) return GB_ERROR_OUT_OF_RANGE;
    return I->rank[b];
}

int gb_get_partials_pool(int instance, void **devicePtr, long long *bytes) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (devicePtr) *devicePtr = I->d_partials;
    if (bytes) *bytes = (long long)I->nbuf * I->cla_stride() * I->elem;
    return GB_SUCCESS;
}

int gb_get_instance_shape(int instance, int *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out[0] = I->ntip;
    out[1] = I->nbuf;
    out[2] = I->S;
    out[3] = I->R;
    out[4] = I->npat;
    return GB_SUCCESS;
}

long long gb_get_launch_count(int instance) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    return I->launches;
}

int gb_synchronize(int instance) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

// ---- engine-side instrumentation (not part of the beagle-equivalent surface) ----
int gb_get_stream(int instance, void **stream) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    *stream = (void *)I->stream;
    return GB_SUCCESS;
}

int gb_set_kernel_timing(int instance, int on) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    resolve_timing(I);
    I->timing = on != 0;
    I->cla_ms = I->edge_ms = 0.0;
    I->cla_launches_timed = I->cla_updates_timed = I->edge_timed = 0;
    return GB_SUCCESS;
}

// out: [0] CLA-kernel ms, [1] CLA launches, [2] pattern-updates, [3] edge ms, [4] edge evals
int gb_get_kernel_timing(int instance, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    resolve_timing(I);
    out[0] = I->cla_ms;
    out[1] = (double)I->cla_launches_timed;
    out[2] = (double)I->cla_updates_timed;
    out[3] = I->edge_ms;
    out[4] = (double)I->edge_timed;
    return GB_SUCCESS;
}

}  // extern "C"
