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
#include "gb_batch.cuh"
#include "gb_batch_mixed.cuh"
#include "gb_common.cuh"
#include "gb_dna.cuh"
#include "gb_eigen.cuh"
#include "gb_graph.cuh"
#include "gb_newton_dna.cuh"
#include "gb_nstate.cuh"
#include "gb_persist.cuh"
#include "gb_persist_mixed.cuh"
#include "gb_pmat.cuh"
#include "gb_tc.cuh"

namespace gb {

static thread_local std::string g_last_error;

struct Instance {
    int device = 0;
    int ntip = 0, nbuf = 0, S = 0, R = 0, npat = 0, npat_pad = 0, neigen = 0, nmat = 0;
    long flags = 0;
    bool mixed = false;
    size_t elem = 8;     // storage bytes an element of the bulk segment (FP64 8, FP32 4, FP32 + extension 5)
    int kpad = 0;        // patterns [0, kpad) stored in FP64 (internal order)
    int kpad_cap = 0;    // FP64 segment size the buffers are laid out for
    int nsm = 148;       // multiprocessors of the device
    int nvb4 = 0;        // 4-state edge evaluations: blocks (= pattern partition) of every
                         // edge kernel, equal to the persistent pass kernel's grid
    long long cla_bytes = 0;
    // host copies in the caller's pattern order and the internal permutation
    // (precision form: patterns with count >= kHeavyCount first, stored in FP64)
    std::vector<uint8_t> h_tips;
    std::vector<int> h_counts, h_cs;
    std::vector<int> perm;  // internal pattern q holds caller pattern perm[q]
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
    double *d_site_d1 = nullptr, *d_site_d2 = nullptr;  // per-site derivatives of the last derivative evaluation
    bool site_deriv_valid = false;
    // pinned result staging
    double *h_result = nullptr;
    int *h_status = nullptr;
    // host state
    std::vector<double> h_rates;
    double pinv = 0.0;
    int has_pinv = 0, last_const = -1;
    std::vector<int> rank;  // per CLA buffer (condlike.h rescaleRank)
    std::vector<char> wide; // per CLA buffer: 1 = FP64 (wide, batched pass only), 2 = its second slot
    long long launches = 0;
    long long bytes = 0;
    bool site_valid = false;
    // optional CLA kernel timing (CUDA events on the instance stream)
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    std::vector<long long> ev_updates;
    std::vector<double> ev_bytes;
    std::vector<double> ev_fp64;  // FP64 instructions of each timed CLA launch
    double cla_ms = 0.0, cla_bytes_timed = 0.0, cla_fp64_timed = 0.0;
    long long cla_launches_timed = 0, cla_updates_timed = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_edge;
    double edge_ms = 0.0;
    long long edge_timed = 0;
    // graph-resident branch-optimisation pass
    double *d_len = nullptr;   // branch length per matrix index (device copy)
    NrSlot *d_slots = nullptr; // Newton state per matrix index
    unsigned long long version = 1;  // bumped by every setter baked into a graph
    unsigned long long graph_key = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_nodes = 0;
    // persistent pass kernel (4 states): command queue and its scratch
    PCmd *d_cmds = nullptr;
    DevOp *d_pops = nullptr;
    size_t cap_cmds = 0, cap_pops = 0;
    GridSync *d_gsync = nullptr;
    double *d_sums2 = nullptr;
    unsigned long long pass_key = 0;
    int use_persistent = 1;
    unsigned long long *d_trace = nullptr;
    int trace_cap = 0;
    // batched candidate pass (gb_batch_newton): queue, results and scratch
    BCmd *d_bcmds = nullptr;
    DevOp *d_bops = nullptr;
    BEntry *d_bentries = nullptr;
    BSlot *d_bslots = nullptr;
    double *d_chunk_sums = nullptr;
    int *d_active = nullptr;  // 2 x cap_bentries, then 2 counters
    size_t cap_bcmds = 0, cap_bops = 0, cap_bentries = 0, cap_bslots = 0, cap_chunk = 0, cap_active = 0;
    int batch_tiles = 0, batch_chunks = 0;  // 0: autotune on the next call
    MEntry *d_mentries = nullptr;  // precision form: spectral coefficients per step
    double *d_coef = nullptr, *d_etab = nullptr;
    int *d_cscale = nullptr;
    size_t cap_mentries = 0, cap_coef = 0, cap_etab = 0, cap_cscale = 0;
    cudaGraph_t bgraph = nullptr;
    cudaGraphExec_t bgraph_exec = nullptr;
    unsigned long long bgraph_key = 0;
    int use_batch_graph = 1;
    int use_tc = 0;  // precision form, 20 / 61 states: CLA updates on the tensor cores
    unsigned char *d_tctab = nullptr;  // per-op P digit tables of a tensor-core level (k_pdigits)
    // model slots, one per eigen index (model_slot_stride doubles each): the
    // instance-wide setters write every slot, gb_set_model_slot one
    std::vector<double> h_mslots;
    double *d_mslots = nullptr;
    double *d_multi = nullptr;  // results of gb_calculate_edges, 3 per edge
    size_t cap_multi = 0;
    // CLA launch shapes chosen by timing (autotune_levels): blocks per SM the
    // per-tree precision 4-state level launch aims at, patterns per block of
    // the n-state CUDA-core CLA kernel; 0 = the built-in choice
    int lvl_target = 0, ns_tp = 0;
    // resident blocks per SM of a kernel at a dynamic shared memory size (queried once)
    struct Occ {
        const void *f;
        size_t smem;
        int blocks;
    };
    std::vector<Occ> occ_cache;
    bool tune_pending = true;
    // scratch of gb_set_eigen_from_rate_matrices, kept between calls
    double *d_eq = nullptr, *d_epi = nullptr;
    EigenJob *d_ejobs = nullptr;
    int *d_esw = nullptr;
    int cap_eig = 0;
    double batch_ms = 0.0;  // CUDA-event time of the timed batched launches
    long long batch_timed = 0;
    // per-phase timing of the batched pass (levels, coefficient passes, Newton /
    // score runs): every launch bracketed by its own events, no graph
    bool phase_timing = false;
    double phase_ms[3] = {0.0, 0.0, 0.0};
    long long phase_launches[3] = {0, 0, 0};

    long long mat_stride() const { return 3LL * R * S * S; }
    long long eig_stride() const { return (long long)S + 2LL * S * S; }
};

static std::mutex g_mu;
static std::vector<Instance *> g_inst;

// precision form: a pattern with at least this count keeps FP64 CLAs (its
// rounding error would be multiplied by the count in the lnL sum)
constexpr int kHeavyCount = 2;

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

// model slot `slot` supplies the state frequencies, category weights and the
// invariant-sites term (slot 0 = the instance-wide model)
static View make_view(Instance *I, int slot = 0) {
    View v;
    v.partials = reinterpret_cast<char *>(I->d_partials);
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
    v.site_d1 = I->d_site_d1;
    v.site_d2 = I->d_site_d2;
    v.cla_bytes = I->cla_bytes;
    v.mat_stride = I->mat_stride();
    v.npat = I->npat;
    v.npat_pad = I->npat_pad;
    v.ntip = I->ntip;
    v.kpad = I->kpad;
    v.has_pinv = I->has_pinv;
    v.rescale_every = 16;
    v.pinv = I->pinv;
    if (slot > 0) {
        const int ms = model_slot_stride(I->S, I->R);
        const double *hs = I->h_mslots.data() + (size_t)slot * ms;
        v.freqs = I->d_mslots + (size_t)slot * ms;
        v.rate_probs = v.freqs + I->S + I->R;
        v.pinv = hs[I->S + 2 * I->R];
        v.has_pinv = hs[I->S + 2 * I->R + 1] != 0.0;
    }
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
template <bool G, bool D>
static void launch_edge4(int R, int grid, cudaStream_t st, const View &v, int pb, int cb, int mat, int tip,
                         int ws) {
    switch (R) {
        case 1: k_edge4<1, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 2: k_edge4<2, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 3: k_edge4<3, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 4: k_edge4<4, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 5: k_edge4<5, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 6: k_edge4<6, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        case 7: k_edge4<7, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
        default: k_edge4<8, G, D><<<grid, kThreads, 0, st>>>(v, pb, cb, mat, tip, ws); break;
    }
}

static size_t ns_cla_smem(const Instance *I, int tp) { return ns_cla_smem_bytes(I->S, I->R, tp); }
// patterns of one warp task of k_cla_ns: tiles are multiples of it
static int ns_pw(const Instance *I) { return I->S <= 20 ? NsTile<20>::PW : NsTile<61>::PW; }
// the largest tile (<= 64 patterns, a power of two: it divides the
// 128-pattern FP64 segment) with at most one warp task per warp that fits 200 KB
static int ns_tp_max(const Instance *I) {
    const int pw = ns_pw(I);
    int tp = 64;
    while (tp > pw && (I->R * (tp / pw) > kThreads / 32 || ns_cla_smem(I, tp) > 200 * 1024)) tp >>= 1;
    return tp;
}
// that tile, or the tuned one rounded up to a power of two of at least the warp task
static int ns_cla_tile(const Instance *I, size_t *smem) {
    int tp = ns_tp_max(I);
    if (I->ns_tp > 0) {
        int t = ns_pw(I);
        while (t < I->ns_tp) t <<= 1;
        tp = std::min(tp, t);
    }
    *smem = ns_cla_smem(I, tp);
    return tp;
}
// the precision form's FP64 pattern segment beside the tensor-core kernel: a
// few hundred patterns, so the smallest tile (many blocks) rather than deep ones
static int ns_seg_tile(const Instance *I, size_t *smem) {
    const int tp = ns_pw(I);
    *smem = ns_cla_smem(I, tp);
    return tp;
}
static void *ns_cla_func(int S, bool garli) {
    if (S <= 20) return garli ? (void *)k_cla_ns<true, 20> : (void *)k_cla_ns<false, 20>;
    return garli ? (void *)k_cla_ns<true, 61> : (void *)k_cla_ns<false, 61>;
}
// blocks per op: at most one resident wave over all ops of the launch, each
// block walking its op's tiles (P staged once per block)
static int occupancy(Instance *I, const void *f, size_t smem) {
    for (const auto &o : I->occ_cache)
        if (o.f == f && o.smem == smem) return o.blocks;
    int occ = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, f, kThreads, smem) != cudaSuccess || occ < 1) occ = 1;
    I->occ_cache.push_back({f, smem, occ});
    return occ;
}
static dim3 ns_cla_grid(Instance *I, void *f, size_t smem, int npat, int tp, int nops) {
    const int occ = occupancy(I, f, smem);
    const int ntiles = (npat + tp - 1) / tp;
    const int per_op = std::max(1, occ * I->nsm / std::max(1, nops));
    return dim3(std::max(1, std::min(ntiles, per_op)), nops);
}
// opt-in dynamic shared memory of the n-state edge kernel (the device's 227 KB
// per block less the kernel's static reduction array)
constexpr int kEdgeSmemMax = 227 * 1024 - 1024;
static void *ns_edge_func(int S, bool garli, bool deriv) {
    if (S <= 20)
        return garli ? (deriv ? (void *)k_edge_ns<true, true, 20> : (void *)k_edge_ns<true, false, 20>)
                     : (deriv ? (void *)k_edge_ns<false, true, 20> : (void *)k_edge_ns<false, false, 20>);
    return garli ? (deriv ? (void *)k_edge_ns<true, true, 61> : (void *)k_edge_ns<true, false, 61>)
                 : (deriv ? (void *)k_edge_ns<false, true, 61> : (void *)k_edge_ns<false, false, 61>);
}
// pattern tile of k_edge_ns (as k_cla_ns: a power of two, at most one warp
// task per warp, the derivative form within 200 KB) and its dynamic shared
// memory (derivative form: the larger)
static int ns_edge_tile(const Instance *I, size_t *smem) {
    const int pw = I->S <= 20 ? NsTile<20, kEdgeQ>::PW : NsTile<61, kEdgeQ>::PW;
    int tp = 64;
    while (tp > pw && (I->R * (tp / pw) > kThreads / 32 || ns_edge_smem_bytes(I->S, I->R, tp, true) > 200 * 1024))
        tp >>= 1;
    // 61 states with 2 categories hold 179 KB of matrices: up to the opt-in limit (kEdgeSmemMax)
    *smem = ns_edge_smem_bytes(I->S, I->R, tp, true);
    return tp;
}
// blocks of an n-state edge evaluation: one resident wave (the derivative
// form's occupancy), so that evaluations with and without derivatives sum
// the same block partials
static int ns_edge_blocks(Instance *I, int tp, size_t smem) {
    const int occ = occupancy(I, ns_edge_func(I->S, !I->mixed, true), smem);
    const int ntiles = (I->npat + tp - 1) / tp;
    return std::max(1, std::min(std::min(ntiles, occ * I->nsm), kMaxScoreBlocks));
}

// tensor-core CLA update (gb_tc.cuh): supported shapes and launch parameters.
// 20 states with up to 4 categories, 61 states with one (the FP32 tiles of
// both children, the digit planes and the output tile must fit one CTA).
static bool tc_supported(const Instance *I) {
    return I->mixed && I->use_tc && ((I->S == 20 && I->R <= 4) || (I->S == 61 && I->R == 1));
}
// the CLA kernel (dynamic shared memory in *smem) and its per-level table
// kernel k_pdigits (*prep)
static void *tc_func(int S, int R, size_t *smem, void **prep = nullptr) {
#define GB_TC(s, r)                                      \
    if (S == s && R == r) {                              \
        *smem = I8Cfg<s, r>::BYTES;                      \
        if (prep) *prep = (void *)k_pdigits<s, r>;       \
        return (void *)k_cla_i8<s, r>;                   \
    }
    GB_TC(20, 1) GB_TC(20, 2) GB_TC(20, 3) GB_TC(20, 4) GB_TC(61, 1)
#undef GB_TC
    *smem = 0;
    return nullptr;
}
// bytes of the per-op tables of a level (k_pdigits output), for any supported shape
constexpr size_t kTcTableBytes = (size_t)kMaxLevelOps * 48 * 1024;
static_assert(I8Cfg<20, 4>::OPB <= 48 * 1024 && I8Cfg<61, 1>::OPB <= 48 * 1024, "tensor-core table slot");
// grid of a tensor-core level launch: tiles per op split so that the level
// fills the SMs about twice over (one CTA per SM at a time; each CTA runs a
// pipeline over its tiles of one op)
static dim3 tc_grid(const Instance *I, int ntiles, int nops) {
    const int want = (2 * I->nsm + nops - 1) / nops;
    return dim3(std::max(1, std::min(ntiles, want)), nops);
}

static void *level4m_ops_func(int R);
static int set_smem_attrs() {
    const int big = 200 * 1024;
    GB_CUDA(cudaFuncSetAttribute(k_eigen_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)eigen_smem_bytes(61)));
    for (int S : {20, 61})
        for (int R = 1; R <= 4; R++) {
            size_t sm = 0;
            void *f = tc_func(S, R, &sm);
            if (f) GB_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        }
    for (int S : {20, 61})
        for (bool g : {true, false})
            GB_CUDA(cudaFuncSetAttribute(ns_cla_func(S, g), cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    for (int S : {20, 61})
        for (bool g : {true, false})
            for (bool d : {true, false})
                GB_CUDA(cudaFuncSetAttribute(ns_edge_func(S, g, d), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kEdgeSmemMax));
    GB_CUDA(cudaFuncSetAttribute(k_pmats, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    for (int R = 1; R <= 8; R++)
        GB_CUDA(cudaFuncSetAttribute(level4m_ops_func(R), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     cp_smem_bytes()));
    GB_CUDA(cudaFuncSetAttribute(k_pmat_len, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    return GB_SUCCESS;
}

static void *pass4_func(int R, bool garli) {
    // precision form: its own kernel (gb_persist_mixed.cuh)
    if (!garli) {
        switch (R) {
            case 1: return (void *)k_pass4m<1>;
            case 2: return (void *)k_pass4m<2>;
            case 3: return (void *)k_pass4m<3>;
            case 4: return (void *)k_pass4m<4>;
            case 5: return (void *)k_pass4m<5>;
            case 6: return (void *)k_pass4m<6>;
            case 7: return (void *)k_pass4m<7>;
            default: return (void *)k_pass4m<8>;
        }
    }
#define GB_CASE(r) \
    case r: return (void *)k_pass4<r, true>;
    switch (R) {
        GB_CASE(1) GB_CASE(2) GB_CASE(3) GB_CASE(4) GB_CASE(5) GB_CASE(6) GB_CASE(7) default : GB_CASE(8)
    }
#undef GB_CASE
}

// grid of a 4-state CLA level: tiles x ops, about 16 resident blocks per SM in total
static dim3 cla4_grid(const Instance *I, int nops) {
    const int G = I->R <= 1 ? 1 : I->R <= 2 ? 2 : I->R <= 4 ? 4 : 8;
    const int ppb = kThreads / G;
    // the precision form's k_cla4m takes kCla4mTiles tiles per block step
    const int ntiles = (I->npat + ppb - 1) / ppb, step = I->mixed ? kCla4mTiles : 1;
    const int want = (16 * I->nsm + nops - 1) / nops;
    return dim3(std::max(1, std::min((ntiles + step - 1) / step, want)), nops);
}

static void *cla4_func(int R, bool garli);

// the precision form's per-tree CLA level (k_level4m_ops: the batched pass's
// prefetched level code): grid (runs of tpi tiles, ops), about four waves of
// four CTAs per SM
static void *level4m_ops_func(int R) {
#define GB_CASE(r) \
    case r: return (void *)k_level4m_ops<r>;
    switch (R) {
        GB_CASE(1) GB_CASE(2) GB_CASE(3) GB_CASE(4) GB_CASE(5) GB_CASE(6) GB_CASE(7) default : GB_CASE(8)
    }
#undef GB_CASE
}
static dim3 level4m_grid(const Instance *I, int nops, int *tpi) {
    const int G = I->R <= 1 ? 1 : I->R <= 2 ? 2 : I->R <= 4 ? 4 : 8;
    const int ctiles = (I->npat + kThreads / G - 1) / (kThreads / G);
    const long long want = (long long)(I->lvl_target > 0 ? I->lvl_target : 16) * I->nsm;  // blocks in the launch
    const long long t = ((long long)ctiles * nops + want - 1) / want;
    *tpi = (int)std::max(1LL, std::min(32LL, t));
    return dim3((ctiles + *tpi - 1) / *tpi, nops);
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
        if (I->S == 4 && I->mixed) {
            int tpi = 1;
            const dim3 grid = level4m_grid(I, L.n, &tpi);
            void *args[] = {&v, &L, &tpi};
            GB_CUDA(cudaLaunchKernel(level4m_ops_func(I->R), grid, dim3(kThreads), args, cp_smem_bytes(),
                                     I->stream));
        } else if (I->S == 4) {
            const dim3 grid = cla4_grid(I, L.n);
            void *args[] = {&v, &L};
            GB_CUDA(cudaLaunchKernel(cla4_func(I->R, !I->mixed), grid, dim3(kThreads), args, 0, I->stream));
        } else {
            size_t smem;
            // precision form on the tensor cores: CUDA cores keep only the FP64 segment
            const bool tc = tc_supported(I);
            const int tp = tc ? ns_seg_tile(I, &smem) : ns_cla_tile(I, &smem);
            const int ns_pat = tc ? std::min(I->kpad, I->npat) : I->npat;
            if (ns_pat > 0) {
                void *f = ns_cla_func(I->S, !I->mixed);
                int R = I->R, plim = ns_pat;
                void *args[] = {&v, &L, &R, (void *)&tp, &plim};
                GB_CUDA(cudaLaunchKernel(f, ns_cla_grid(I, f, smem, ns_pat, tp, L.n), dim3(kThreads), args, smem,
                                         I->stream));
            }
            int first = I->kpad / kTcM, nt = I->npat_pad / kTcM - first;
            if (tc && nt > 0) {
                size_t tsm = 0;
                void *prep = nullptr;
                void *f = tc_func(I->S, I->R, &tsm, &prep);
                const unsigned char *tab = I->d_tctab;
                void *pargs[] = {&v, &L, (void *)&tab};
                GB_CUDA(cudaLaunchKernel(prep, dim3(L.n), dim3(kThreads), pargs, 0, I->stream));
                void *args[] = {&v, &L, (void *)&first, (void *)&nt, (void *)&tab};
                GB_CUDA(cudaLaunchKernel(f, tc_grid(I, nt, L.n), dim3(kTcThreads), args, tsm, I->stream));
            }
        }
        int rc = check_launch(I);
        if (rc) return rc;
        if (I->timing) {
            cudaEventRecord(e1, I->stream);
            I->ev.emplace_back(e0, e1);
            I->ev_updates.push_back((long long)L.n * I->npat);
            // algorithmic bytes per pattern: internal-internal 3*R*S*b + 12,
            // internal-tip 2*R*S*b + 9, tip-tip R*S*b + 6 (children read once, dest written once)
            const double rsb = (double)I->R * I->S * I->elem;
            double b = 0.0;
            for (int i = 0; i < L.n; i++)
                b += L.op[i].kind == kIntInt ? 3 * rsb + 12 : L.op[i].kind == kIntTip ? 2 * rsb + 9 : rsb + 6;
            I->ev_bytes.push_back(b * I->npat);
            // FP64 instructions per pattern of the n-state CUDA-core kernel: per output
            // (rate, from) S products and S sums per internal child (one fused
            // instruction each in the precision form) and one product; 4-state
            // kernels are not counted
            double f = 0.0;
            if (I->S != 4) {
                const double per = I->mixed ? 1.0 : 2.0, S = I->S, RS = (double)I->R * I->S;
                for (int i = 0; i < L.n; i++) {
                    const int nint = L.op[i].kind == kIntInt ? 2 : L.op[i].kind == kIntTip ? 1 : 0;
                    f += RS * (nint * per * S + 1.0);
                }
                const bool tc = tc_supported(I);
                const int ns_pat = tc ? std::min(I->kpad, I->npat) : I->npat;
                f *= ns_pat;
            }
            I->ev_fp64.push_back(f);
        }
    }
    return GB_SUCCESS;
}

// Launch shapes by timing, on the first op list large enough to time (>= 2
// levels, >= 2^17 pattern-updates): each candidate runs the whole list twice,
// the second run timed; the fastest is kept.  Every run computes the same
// values from the same inputs (each pattern's arithmetic does not depend on
// the shape), so the list's results are in place afterwards.
static int autotune_levels(Instance *I, const std::vector<std::vector<DevOp>> &levels, int rescaleEvery) {
    I->tune_pending = false;
    std::vector<int> cand;
    int *knob = nullptr;
    if (I->S == 4 && I->mixed) {
        cand = {4, 8, 16, 32};
        knob = &I->lvl_target;
    } else if (I->S != 4 && !tc_supported(I)) {
        for (int tp = ns_pw(I); tp <= ns_tp_max(I); tp *= 2) cand.push_back(tp);
        knob = &I->ns_tp;
    }
    auto run = [&]() -> int {
        for (const auto &lv : levels) {
            int rc = launch_level(I, lv, rescaleEvery);
            if (rc) return rc;
        }
        return GB_SUCCESS;
    };
    if (cand.size() < 2) return run();
    const bool timing = I->timing;
    I->timing = false;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int pick = cand[0], rc = GB_SUCCESS;
    for (int c : cand) {
        *knob = c;
        if ((rc = run())) break;
        cudaEventRecord(e0, I->stream);
        if ((rc = run())) break;
        cudaEventRecord(e1, I->stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = GB_ERROR_GENERAL;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    I->timing = timing;
    *knob = pick;
    I->graph_key = 0;  // a captured pass graph holds the old shapes
    return rc;
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
        I->cla_bytes_timed += I->ev_bytes[i];
        I->cla_fp64_timed += I->ev_fp64[i];
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
    I->ev_bytes.clear();
    I->ev_fp64.clear();
    I->ev_edge.clear();
}

}  // namespace gb

using namespace gb;

// Lets the library's other translation units report through gb_last_error().
void gb_internal_set_last_error(const std::string &msg) { g_last_error = msg; }

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
    // the faster CLA path of the precision form as measured on B200: tensor
    // cores for 61 states, the CUDA-core FP64 kernel for 20
    I->use_tc = stateCount == 61 ? 1 : 0;
    I->flags = I->mixed ? GB_FLAG_MIXED_FP32 : GB_FLAG_PLAIN_FP64;
    I->elem = I->mixed ? (stateCount == 4 ? 5 : 4) : 8;  // the 4-state FP32 segment carries extension bytes
    I->rank.assign(partialsBufferCount, 0);
    I->wide.assign(partialsBufferCount, 0);
    I->h_rates.assign(categoryCount, 1.0);
    // FP64 segment: everything in the plain form; in the precision form room for
    // max(128, npat/32) heavy patterns (rounded to the 128-pattern tile)
    if (I->mixed) {
        const int cap = std::max(128, (I->npat_pad / 32 + 127) / 128 * 128);
        I->kpad_cap = std::min(cap, I->npat_pad);
        I->kpad = 0;
    } else {
        I->kpad_cap = I->kpad = I->npat_pad;
    }
    {
        // FP32 segment of the 4-state precision form: 4 bytes an element plus
        // one extension byte (cla_ext)
        const long long RS = (long long)I->R * I->S;
        const long long f32 = (I->mixed && I->S == 4) ? 5 : 4;
        I->cla_bytes = (long long)I->kpad_cap * RS * 8 + (long long)(I->npat_pad - I->kpad_cap) * RS * f32;
        I->cla_bytes = (I->cla_bytes + 255) / 256 * 256;
    }
    I->h_tips.assign((size_t)tipCount * patternCount, stateCount == 4 ? 15 : stateCount);
    I->h_counts.assign(patternCount, 1);
    I->h_cs.assign(patternCount, -1);
    I->perm.resize(patternCount);
    for (int q = 0; q < patternCount; q++) I->perm[q] = q;
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
    cudaDeviceGetAttribute(&I->nsm, cudaDevAttrMultiProcessorCount, resourceNumber);
    if (stateCount == 4) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass4_func(categoryCount, !I->mixed), kThreads, 0);
        I->nvb4 = std::min(kMaxScoreBlocks, std::max(1, per_sm) * I->nsm);
    }
    const size_t P = I->npat_pad;
    const size_t cla_bytes = (size_t)I->nbuf * I->cla_bytes;
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
        {(void **)&I->d_site_d1, P * sizeof(double)},
        {(void **)&I->d_site_d2, P * sizeof(double)},
        {(void **)&I->d_len, (size_t)I->nmat * sizeof(double)},
        {(void **)&I->d_slots, (size_t)I->nmat * sizeof(NrSlot)},
        {(void **)&I->d_gsync, sizeof(GridSync)},
        {(void **)&I->d_sums2, (size_t)2 * 3 * kMaxScoreBlocks * sizeof(double)},
        {(void **)&I->d_tctab, (I->mixed && I->S != 4) ? kTcTableBytes : (size_t)16},
        {(void **)&I->d_mslots, (size_t)I->neigen * model_slot_stride(I->S, I->R) * sizeof(double)},
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
    {
        // model slots: unit rates and weights 1/R, uniform frequencies, no pinv
        const int ms = model_slot_stride(I->S, I->R);
        I->h_mslots.assign((size_t)I->neigen * ms, 0.0);
        for (int e = 0; e < I->neigen; e++) {
            double *sl = I->h_mslots.data() + (size_t)e * ms;
            for (int i = 0; i < I->S; i++) sl[i] = 1.0 / I->S;
            for (int r = 0; r < I->R; r++) {
                sl[I->S + r] = 1.0;
                sl[I->S + I->R + r] = 1.0 / I->R;
            }
        }
        cudaMemcpyAsync(I->d_mslots, I->h_mslots.data(), I->h_mslots.size() * sizeof(double),
                        cudaMemcpyHostToDevice, I->stream);
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
    cudaMemsetAsync(I->d_const, 0xff, P * sizeof(int), I->stream);
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
    if (I->graph_exec) cudaGraphExecDestroy(I->graph_exec);
    if (I->graph) cudaGraphDestroy(I->graph);
    void *ptrs[] = {I->d_partials, I->d_scalers, I->d_tips, I->d_counts, I->d_const, I->d_mats,
                    I->d_eigen, I->d_freqs, I->d_rates, I->d_rprobs, I->d_status, I->d_block_sums,
                    I->d_result, I->d_site_lnl, I->d_site_d1, I->d_site_d2, I->d_len, I->d_slots, I->d_gsync, I->d_sums2,
                    I->d_cmds, I->d_pops, I->d_bcmds, I->d_bops, I->d_bentries, I->d_bslots,
                    I->d_chunk_sums, I->d_active, I->d_mentries, I->d_coef, I->d_etab, I->d_cscale,
                    I->d_tctab, I->d_mslots, I->d_multi, I->d_eq, I->d_epi, I->d_ejobs, I->d_esw};
    if (I->bgraph_exec) cudaGraphExecDestroy(I->bgraph_exec);
    if (I->bgraph) cudaGraphDestroy(I->bgraph);
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

}  // extern "C"

namespace gb {

static int upload_tip(Instance *I, int t) {
    std::vector<uint8_t> row(I->npat);
    const uint8_t *src = I->h_tips.data() + (size_t)t * I->npat;
    for (int q = 0; q < I->npat; q++) row[q] = src[I->perm[q]];
    GB_CUDA(cudaMemcpyAsync(I->d_tips + (size_t)t * I->npat_pad, row.data(), I->npat, cudaMemcpyHostToDevice,
                            I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

static int upload_patterns(Instance *I) {
    std::vector<int> c(I->npat), cs(I->npat);
    for (int q = 0; q < I->npat; q++) {
        c[q] = I->h_counts[I->perm[q]];
        cs[q] = I->h_cs[I->perm[q]];
    }
    GB_CUDA(cudaMemcpyAsync(I->d_counts, c.data(), I->npat * sizeof(int), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaMemcpyAsync(I->d_const, cs.data(), I->npat * sizeof(int), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

// precision form: patterns with count >= kHeavyCount go first (largest counts
// first if they exceed the FP64 segment), everything else keeps its order
// write column [off, off + n) of every model slot (or of slot `only`) and upload the table
static int set_slot_columns(Instance *I, int off, int n, const double *vals, int only = -1) {
    const int ms = model_slot_stride(I->S, I->R);
    for (int e = 0; e < I->neigen; e++)
        if (only < 0 || e == only) std::memcpy(I->h_mslots.data() + (size_t)e * ms + off, vals, n * sizeof(double));
    GB_CUDA(cudaMemcpyAsync(I->d_mslots, I->h_mslots.data(), I->h_mslots.size() * sizeof(double),
                            cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

static void make_permutation(Instance *I) {
    std::vector<int> heavy, light;
    for (int q = 0; q < I->npat; q++) (I->h_counts[q] >= kHeavyCount ? heavy : light).push_back(q);
    if ((int)heavy.size() > I->kpad_cap) {
        std::stable_sort(heavy.begin(), heavy.end(),
                         [&](int a, int b) { return I->h_counts[a] > I->h_counts[b]; });
        for (size_t i = I->kpad_cap; i < heavy.size(); i++) light.push_back(heavy[i]);
        heavy.resize(I->kpad_cap);
        std::sort(light.begin(), light.end());
    }
    I->kpad = heavy.empty() ? 0 : std::min(I->kpad_cap, ((int)heavy.size() + 127) / 128 * 128);
    I->perm = heavy;
    I->perm.insert(I->perm.end(), light.begin(), light.end());
}

}  // namespace gb

extern "C" {

int gb_set_tip_states(int instance, int tipIndex, const unsigned char *codes) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
    if (tipIndex < 0 || tipIndex >= I->ntip || !codes) return GB_ERROR_OUT_OF_RANGE;
    const int miss = I->S == 4 ? 15 : I->S;
    for (int p = 0; p < I->npat; p++)
        if (I->S == 4 ? (codes[p] & ~15) != 0 : codes[p] > miss) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    std::memcpy(I->h_tips.data() + (size_t)tipIndex * I->npat, codes, I->npat);
    return upload_tip(I, tipIndex);
}

int gb_set_pattern_weights(int instance, const int *counts) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
    for (int p = 0; p < I->npat; p++)
        if (counts[p] < 0) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    I->h_counts.assign(counts, counts + I->npat);
    if (I->mixed) {
        const std::vector<int> old = I->perm;
        make_permutation(I);
        if (old != I->perm) {
            for (int t = 0; t < I->ntip; t++) {
                int rc = upload_tip(I, t);
                if (rc) return rc;
            }
        }
    }
    return upload_patterns(I);
}

int gb_set_constant_patterns(int instance, int lastConst, const int *constStates) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
    if (lastConst >= I->npat || lastConst < -1) return GB_ERROR_OUT_OF_RANGE;
    for (int p = 0; p <= lastConst; p++)
        if (constStates[p] < 0 || constStates[p] > (I->S == 4 ? 15 : I->S - 1)) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    I->last_const = lastConst;
    for (int p = 0; p < I->npat; p++) I->h_cs[p] = p <= lastConst ? constStates[p] : -1;
    return upload_patterns(I);
}

int gb_set_state_frequencies(int instance, const double *freqs) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(I->d_freqs, freqs, I->S * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return set_slot_columns(I, 0, I->S, freqs);
}

int gb_set_category_rates(int instance, const double *rates) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
    cudaSetDevice(I->device);
    I->h_rates.assign(rates, rates + I->R);
    GB_CUDA(cudaMemcpyAsync(I->d_rates, rates, I->R * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return set_slot_columns(I, I->S, I->R, rates);
}

int gb_set_category_weights(int instance, const double *weights) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(I->d_rprobs, weights, I->R * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return set_slot_columns(I, I->S + I->R, I->R, weights);
}

int gb_set_invariant_sites(int instance, double pinv, int hasPinv) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
    if (!(pinv >= 0.0 && pinv < 1.0)) return GB_ERROR_OUT_OF_RANGE;
    I->pinv = pinv;
    I->has_pinv = hasPinv ? 1 : 0;
    cudaSetDevice(I->device);
    const double pv[2] = {pinv, hasPinv ? 1.0 : 0.0};
    return set_slot_columns(I, I->S + 2 * I->R, 2, pv);
}

// One model slot (the parameters read with eigen index eigenIndex): state
// frequencies, category rates and weights, invariant sites.  Slot 0 is also
// the instance-wide model of the kernels that take no eigen index; the other
// slots are left as they are.
int gb_set_model_slot(int instance, int eigenIndex, const double *freqs, const double *rates,
                      const double *weights, double pinv, int hasPinv) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (eigenIndex < 0 || eigenIndex >= I->neigen || !freqs || !rates || !weights || !(pinv >= 0.0 && pinv < 1.0))
        return GB_ERROR_OUT_OF_RANGE;
    I->version++;
    cudaSetDevice(I->device);
    const int S = I->S, R = I->R, ms = model_slot_stride(S, R);
    if (eigenIndex == 0) {
        I->h_rates.assign(rates, rates + R);
        I->pinv = pinv;
        I->has_pinv = hasPinv ? 1 : 0;
        GB_CUDA(cudaMemcpyAsync(I->d_freqs, freqs, S * sizeof(double), cudaMemcpyHostToDevice, I->stream));
        GB_CUDA(cudaMemcpyAsync(I->d_rates, rates, R * sizeof(double), cudaMemcpyHostToDevice, I->stream));
        GB_CUDA(cudaMemcpyAsync(I->d_rprobs, weights, R * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    }
    double *sl = I->h_mslots.data() + (size_t)eigenIndex * ms;
    std::memcpy(sl, freqs, S * sizeof(double));
    std::memcpy(sl + S, rates, R * sizeof(double));
    std::memcpy(sl + S + R, weights, R * sizeof(double));
    sl[S + 2 * R] = pinv;
    sl[S + 2 * R + 1] = hasPinv ? 1.0 : 0.0;
    return set_slot_columns(I, 0, ms, sl, eigenIndex);
}

int gb_set_eigen_decomposition(int instance, int eigenIndex, const double *U, const double *Uinv,
                               const double *lambda) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->version++;
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
        const size_t smem = pmat_smem_bytes(I->S, I->R);
        k_pmats<<<dim3(T.n, pmat_chunks(I->S, I->R)), kThreads, smem, I->stream>>>(
            I->d_eigen, I->eig_stride(), I->S, I->R, I->d_mslots, T, I->d_mats, I->mat_stride());
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

}  // extern "C"

namespace gb {

// Normalise, validate and level a list of ClaOperations; applies GARLI's rank
// rule (tree.cpp:7665-8598) to the instance's rank table as the ops would
// execute and returns the per-level device op lists.
static int prepare_ops(Instance *I, const gb_cla_operation *ops, int count, int rescaleEvery,
                       std::vector<std::vector<DevOp>> &levels, bool allow_wide = false) {
    levels.clear();
    if (count <= 0) return GB_SUCCESS;
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return ops[a].opDepLevel < ops[b].opDepLevel; });
    const int nt = I->ntip, nb = I->nbuf;
    auto is_tip = [&](int b) { return b >= 0 && b < nt; };
    auto is_cla = [&](int b) { return b >= nt && b < nt + nb; };
    int cur = ops[order[0]].opDepLevel;
    levels.emplace_back();
    for (int k = 0; k < count; k++) {
        const gb_cla_operation &o = ops[order[k]];
        if (o.opDepLevel != cur) {
            cur = o.opDepLevel;
            levels.emplace_back();
        }
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
        d.wide = 0;
        {
            const char wd = I->wide[dest], w1 = is_cla(c1) ? I->wide[c1 - nt] : 0, w2 = is_cla(c2) ? I->wide[c2 - nt] : 0;
            if (wd == 2 || w1 == 2 || w2 == 2) return GB_ERROR_OUT_OF_RANGE;  // the second slot of a wide buffer
            d.wide = (wd ? kWideDest : 0) | (w1 ? kWideC1 : 0) | (w2 ? kWideC2 : 0);
            if (d.wide && !allow_wide) {
                g_last_error = "FP64 (wide) buffers are read and written by gb_batch_newton only";
                return GB_ERROR_NO_IMPLEMENTATION;
            }
        }
        d.p1 = p1;
        d.p2 = p2;
        d.rescale = (!I->mixed && rank >= rescaleEvery) ? 1 : 0;
        I->rank[dest] = d.rescale ? 0 : rank;
        levels.back().push_back(d);
    }
    return GB_SUCCESS;
}

}  // namespace gb

extern "C" {

int gb_update_partials(int instance, const gb_cla_operation *ops, int count, int rescaleEvery) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (count < 0) return GB_ERROR_OUT_OF_RANGE;
    if (count == 0) return GB_SUCCESS;
    cudaSetDevice(I->device);
    std::vector<std::vector<DevOp>> levels;
    int rc = prepare_ops(I, ops, count, rescaleEvery, levels);
    if (rc) return rc;
    if (I->tune_pending && levels.size() >= 2 && (long long)count * I->npat >= (1LL << 17))
        return autotune_levels(I, levels, rescaleEvery);
    for (auto &lv : levels) {
        rc = launch_level(I, lv, rescaleEvery);
        if (rc) return rc;
    }
    return GB_SUCCESS;
}

int gb_set_cla_tuning(int instance, int levelBlocksPerSm, int nstateTilePatterns) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (levelBlocksPerSm < -1 || levelBlocksPerSm > 64 || nstateTilePatterns < -1 || nstateTilePatterns > 64)
        return GB_ERROR_OUT_OF_RANGE;
    if (levelBlocksPerSm > 0) I->lvl_target = levelBlocksPerSm;
    if (nstateTilePatterns > 0) I->ns_tp = nstateTilePatterns;
    I->tune_pending = levelBlocksPerSm == 0 || nstateTilePatterns == 0;
    I->graph_key = 0;
    return GB_SUCCESS;
}

int gb_get_cla_tuning(int instance, int *out3) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    size_t smem;
    out3[0] = I->lvl_target > 0 ? I->lvl_target : 16;
    out3[1] = ns_cla_tile(I, &smem);
    out3[2] = I->tune_pending ? 1 : 0;
    return GB_SUCCESS;
}

// enqueue one edge evaluation under model slot `slot`; its (lnL, d1, d2) go to dres
static int edge_enqueue(Instance *I, const gb_scoring_operation *op, int slot, double *dres) {
    const int nt = I->ntip;
    const int pb = op->childClaIndex1 - nt;
    const int cb = op->childClaIndex2;
    if (pb < 0 || pb >= I->nbuf || cb < 0 || cb >= nt + I->nbuf || op->transMatIndex < 0 ||
        op->transMatIndex >= I->nmat || slot < 0 || slot >= I->neigen)
        return GB_ERROR_OUT_OF_RANGE;
    const int tip = cb < nt;
    const int cidx = tip ? cb : cb - nt;
    View v = make_view(I, slot);
    const bool D = op->derivatives != 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (I->timing) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, I->stream);
    }
    int nblocks;
    if (I->S == 4) {
        nblocks = I->nvb4;
        if (I->mixed) {
            if (D) launch_edge4<false, true>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
            else launch_edge4<false, false>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
        } else {
            if (D) launch_edge4<true, true>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
            else launch_edge4<true, false>(I->R, nblocks, I->stream, v, pb, cidx, op->transMatIndex, tip, 1);
        }
    } else {
        size_t smem;
        int tp = ns_edge_tile(I, &smem);
        nblocks = ns_edge_blocks(I, tp, smem);
        int pbi = pb, cbi = cidx, mat = op->transMatIndex, tipi = tip, ws = 1, R = I->R;
        void *args[] = {&v, &pbi, &cbi, &mat, &tipi, &ws, &R, &tp};
        GB_CUDA(cudaLaunchKernel(ns_edge_func(I->S, !I->mixed, D), dim3(nblocks), dim3(kThreads), args, smem,
                                 I->stream));
    }
    int rc = check_launch(I);
    if (rc) return rc;
    k_reduce3<<<1, kThreads, 0, I->stream>>>(I->d_block_sums, nblocks, dres);
    rc = check_launch(I);
    if (rc) return rc;
    if (I->timing) {
        cudaEventRecord(e1, I->stream);
        I->ev_edge.emplace_back(e0, e1);
    }
    I->site_valid = true;
    I->site_deriv_valid = D;
    return GB_SUCCESS;
}

// status word of the work enqueued so far (read after a stream synchronisation)
static int edge_status(Instance *I) {
    if (*I->h_status & kStatusTcRange) {
        // a product maximum below the tensor-core path's range: the CLAs are
        // recomputed on the CUDA cores (the tree drivers redo the score on
        // GB_ERROR_RESCALE_RETRY; the precision form's scaling ignores rescaleEvery)
        I->use_tc = 0;
        I->graph_key = 0;
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        return GB_ERROR_RESCALE_RETRY;
    }
    if (*I->h_status & kStatusBarrierTimeout) {
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        g_last_error = "CLA level: a prefetch wait exceeded its bound";
        return GB_ERROR_GENERAL;
    }
    if (*I->h_status & kStatusTcTimeout) {
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        g_last_error = "tensor-core CLA update: an mbarrier wait exceeded its bound";
        return GB_ERROR_GENERAL;
    }
    if (*I->h_status & kStatusRescaleRetry) {
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        return GB_ERROR_RESCALE_RETRY;
    }
    return GB_SUCCESS;
}

static int edge_impl(Instance *I, const gb_scoring_operation *op, double *out, bool sync) {
    int rc = edge_enqueue(I, op, 0, I->d_result);
    if (rc || !sync) return rc;
    const bool D = op->derivatives != 0;
    GB_CUDA(cudaMemcpyAsync(I->h_result, I->d_result, 3 * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaMemcpyAsync(I->h_status, I->d_status, sizeof(int), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    out[0] = I->h_result[0];
    out[1] = D ? I->h_result[1] : 0.0;
    out[2] = D ? I->h_result[2] : 0.0;
    if ((rc = edge_status(I))) return rc;
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

// count edge evaluations, edge k under model slot modelSlots[k] (all slot 0
// when modelSlots is NULL), with one synchronisation; out[3k .. 3k+2]
int gb_calculate_edges(int instance, const gb_scoring_operation *ops, const int *modelSlots, int count,
                       double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!ops || !out || count < 1) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    if ((size_t)count * 3 > I->cap_multi) {
        cudaFree(I->d_multi);
        I->d_multi = nullptr;
        I->cap_multi = 0;
        if (cudaMalloc(&I->d_multi, (size_t)count * 3 * sizeof(double)) != cudaSuccess) {
            g_last_error = "gb_calculate_edges: cudaMalloc failed";
            return GB_ERROR_OUT_OF_MEMORY;
        }
        I->cap_multi = (size_t)count * 3;
    }
    for (int k = 0; k < count; k++) {
        int rc = edge_enqueue(I, ops + k, modelSlots ? modelSlots[k] : 0, I->d_multi + 3 * k);
        if (rc) return rc;
    }
    std::vector<double> res((size_t)count * 3);
    GB_CUDA(cudaMemcpyAsync(res.data(), I->d_multi, res.size() * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaMemcpyAsync(I->h_status, I->d_status, sizeof(int), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    int rc = edge_status(I);
    if (rc) return rc;
    for (int k = 0; k < count; k++) {
        const bool D = ops[k].derivatives != 0;
        out[3 * k] = res[3 * k];
        out[3 * k + 1] = D ? res[3 * k + 1] : 0.0;
        out[3 * k + 2] = D ? res[3 * k + 2] : 0.0;
        if (!std::isfinite(out[3 * k])) return GB_ERROR_FLOATING_POINT;
    }
    return GB_SUCCESS;
}

int gb_get_site_log_likelihoods(int instance, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!I->site_valid) return GB_ERROR_GENERAL;
    cudaSetDevice(I->device);
    std::vector<double> tmp(I->npat);
    GB_CUDA(cudaMemcpyAsync(tmp.data(), I->d_site_lnl, I->npat * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    for (int q = 0; q < I->npat; q++) out[I->perm[q]] = tmp[q];
    return GB_SUCCESS;
}

// beagleGetSiteDerivatives (subsetcalculationmanager.cpp:440, OutputBeagleSiteValues)
int gb_get_site_derivatives(int instance, double *outFirst, double *outSecond) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!outFirst || !outSecond) return GB_ERROR_OUT_OF_RANGE;
    if (!I->site_deriv_valid) return GB_ERROR_GENERAL;
    cudaSetDevice(I->device);
    std::vector<double> a(I->npat), b(I->npat);
    GB_CUDA(cudaMemcpyAsync(a.data(), I->d_site_d1, I->npat * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaMemcpyAsync(b.data(), I->d_site_d2, I->npat * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    for (int q = 0; q < I->npat; q++) {
        outFirst[I->perm[q]] = a[q];
        outSecond[I->perm[q]] = b[q];
    }
    return GB_SUCCESS;
}

int gb_get_partials(int instance, int bufferIndex, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    const int b = bufferIndex - I->ntip;
    if (b < 0 || b >= I->nbuf) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    const int RS = I->R * I->S;
    std::vector<char> raw(I->cla_bytes);
    GB_CUDA(cudaMemcpyAsync(raw.data(), (const char *)I->d_partials + (size_t)b * I->cla_bytes, I->cla_bytes,
                            cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    const double *d64 = reinterpret_cast<const double *>(raw.data());
    const float *d32 = reinterpret_cast<const float *>(raw.data() + (size_t)I->kpad * RS * 8);
    if (I->wide[b] == 1) {  // FP64 throughout, over two buffer slots
        std::vector<double> wraw((size_t)I->npat * RS);
        GB_CUDA(cudaMemcpyAsync(wraw.data(), (const char *)I->d_partials + (size_t)b * I->cla_bytes,
                                wraw.size() * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        for (int q = 0; q < I->npat; q++)
            std::memcpy(out + (size_t)I->perm[q] * RS, wraw.data() + (size_t)q * RS, RS * sizeof(double));
        return GB_SUCCESS;
    }
    // 4-state precision form: each FP32 element's extension byte (cla_ext)
    const bool ext = I->mixed && I->S == 4;
    const unsigned char *e8 =
        reinterpret_cast<const unsigned char *>(raw.data() + (size_t)I->kpad * RS * 8 + (size_t)(I->npat_pad - I->kpad) * RS * 4);
    for (int q = 0; q < I->npat; q++) {
        double *dst = out + (size_t)I->perm[q] * RS;
        for (int k = 0; k < RS; k++) {
            if (q < I->kpad) {
                dst[k] = d64[(size_t)q * RS + k];
                continue;
            }
            const float hi = d32[(size_t)(q - I->kpad) * RS + k];
            dst[k] = hi;
            if (ext) {  // the device's ext_value: the float word's fields and the byte as a double
                uint32_t w;
                std::memcpy(&w, &hi, 4);
                const uint64_t E = (w >> 23) & 0xffu;
                const uint64_t b = ((E + 896u) << 52) | ((uint64_t)(w & 0x7fffffu) << 29) |
                                   ((uint64_t)e8[(size_t)(q - I->kpad) * RS + k] << 21);
                double x = 0.0;
                if (E) std::memcpy(&x, &b, 8);
                dst[k] = x;
            }
        }
    }
    return GB_SUCCESS;
}

int gb_get_scale_factors(int instance, int bufferIndex, int *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    const int b = bufferIndex - I->ntip;
    if (b < 0 || b >= I->nbuf) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    std::vector<int> tmp(I->npat);
    GB_CUDA(cudaMemcpyAsync(tmp.data(), I->d_scalers + (size_t)b * I->npat_pad, I->npat * sizeof(int),
                            cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    for (int q = 0; q < I->npat; q++) out[I->perm[q]] = tmp[q];
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
    if (bytes) *bytes = (long long)I->nbuf * I->cla_bytes;
    return GB_SUCCESS;
}

int gb_get_instance_capacity(int instance, int *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out[0] = I->nbuf;
    out[1] = I->nmat;
    out[2] = I->neigen;
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
    I->cla_ms = I->edge_ms = I->cla_bytes_timed = I->cla_fp64_timed = 0.0;
    I->cla_launches_timed = I->cla_updates_timed = I->edge_timed = 0;
    return GB_SUCCESS;
}

// out: [0] CLA-kernel ms, [1] CLA launches, [2] pattern-updates, [3] edge ms, [4] edge evals,
//      [5] algorithmic bytes of the timed CLA launches
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
    out[5] = I->cla_bytes_timed;
    out[6] = I->cla_fp64_timed;
    return GB_SUCCESS;
}

}  // extern "C"

// ===========================================================================
// Graph-resident branch-optimisation pass (OptimizeAllBranches on the device)
// ===========================================================================
namespace gb {

static unsigned long long fnv(unsigned long long h, const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// the plain form's k_cla4 (GARLI's rescaling) or the precision form's k_cla4m
static void *cla4_func(int R, bool garli) {
#define GB_CASE(r) \
    case r: return garli ? (void *)k_cla4<r, true> : (void *)k_cla4m<r>;
    switch (R) {
        GB_CASE(1) GB_CASE(2) GB_CASE(3) GB_CASE(4) GB_CASE(5) GB_CASE(6) GB_CASE(7) default : GB_CASE(8)
    }
#undef GB_CASE
}
static void *edge4_deriv_func(int R, bool garli) {
#define GB_CASE(r) \
    case r: return garli ? (void *)k_edge4<r, true, true> : (void *)k_edge4<r, false, true>;
    switch (R) {
        GB_CASE(1) GB_CASE(2) GB_CASE(3) GB_CASE(4) GB_CASE(5) GB_CASE(6) GB_CASE(7) default : GB_CASE(8)
    }
#undef GB_CASE
}

struct GraphBuilder {
    cudaGraph_t g;
    int nodes = 0;
    dim3 block = dim3(kThreads);  // block size of the next node
    int add(cudaGraph_t graph, cudaGraphNode_t *prev, void *func, dim3 grid, size_t smem, void **args) {
        cudaKernelNodeParams kp = {};
        kp.func = func;
        kp.gridDim = grid;
        kp.blockDim = block;
        kp.sharedMemBytes = (unsigned)smem;
        kp.kernelParams = args;
        cudaGraphNode_t n;
        cudaError_t e = cudaGraphAddKernelNode(&n, graph, *prev ? prev : nullptr, *prev ? 1 : 0, &kp);
        if (e != cudaSuccess) {
            g_last_error = std::string("cudaGraphAddKernelNode: ") + cudaGetErrorString(e);
            return GB_ERROR_GENERAL;
        }
        *prev = n;
        nodes++;
        return GB_SUCCESS;
    }
};

static void *nr_iter4_func(int R, bool garli) {
#define GB_CASE(r) \
    case r: return garli ? (void *)k_nr_iter4<r, true> : (void *)k_nr_iter4<r, false>;
    switch (R) {
        GB_CASE(1) GB_CASE(2) GB_CASE(3) GB_CASE(4) GB_CASE(5) GB_CASE(6) GB_CASE(7) default : GB_CASE(8)
    }
#undef GB_CASE
}

// levels[b] = the prepared (levelled, rank-flagged) CLA updates of branch b
static int build_pass_graph(Instance *I, const gb_nr_branch *br, int nbr,
                            const std::vector<std::vector<std::vector<DevOp>>> &levels, int rescaleEvery,
                            NrParams prm) {
    if (I->graph_exec) cudaGraphExecDestroy(I->graph_exec);
    if (I->graph) cudaGraphDestroy(I->graph);
    I->graph_exec = nullptr;
    I->graph = nullptr;
    GraphBuilder B;
    GB_CUDA(cudaGraphCreate(&B.g, 0));
    I->graph = B.g;
    View v = make_view(I);
    v.rescale_every = rescaleEvery;
    cudaGraphNode_t prev = nullptr;
    const bool dna = I->S == 4;
    const bool garli = !I->mixed;
    size_t ns_smem = 0, ns_edge_smem = 0;
    int ns_tp = 0, ns_edge_tp = 0;
    if (!dna) {
        ns_tp = ns_cla_tile(I, &ns_smem);
        ns_edge_tp = ns_edge_tile(I, &ns_edge_smem);
    }
    const int nblocks = dna ? I->nvb4 : ns_edge_blocks(I, ns_edge_tp, ns_edge_smem);
    const size_t pmat_smem = pmat_smem_bytes(I->S, I->R);
    int rc;
    {
        int n = I->nmat;
        void *args[] = {&I->d_slots, &n};
        rc = B.add(B.g, &prev, (void *)k_nr_reset, dim3((n + kThreads - 1) / kThreads), 0, args);
        if (rc) return rc;
    }
    for (int b = 0; b < nbr; b++) {
        const gb_nr_branch &nb = br[b];
        for (auto &lv : levels[b]) {
            for (size_t c = 0; c < lv.size(); c += kMaxLevelOps) {
                LevelOps L;
                L.n = (int)std::min<size_t>(kMaxLevelOps, lv.size() - c);
                for (int i = 0; i < L.n; i++) L.op[i] = lv[c + i];
                if (dna && !garli) {
                    int tpi = 1;
                    const dim3 grid = level4m_grid(I, L.n, &tpi);
                    void *args[] = {&v, &L, &tpi};
                    rc = B.add(B.g, &prev, level4m_ops_func(I->R), grid, cp_smem_bytes(), args);
                } else if (dna) {
                    void *args[] = {&v, &L};
                    rc = B.add(B.g, &prev, cla4_func(I->R, garli), cla4_grid(I, L.n), 0, args);
                } else {
                    int S = I->S, R = I->R, tp = ns_tp;
                    size_t smem = ns_smem;
                    const bool tc = tc_supported(I);
                    if (tc) tp = ns_seg_tile(I, &smem);
                    const int ns_pat = tc ? std::min(I->kpad, I->npat) : I->npat;
                    if (ns_pat > 0) {
                        int plim = ns_pat;
                        void *f = ns_cla_func(S, garli);
                        void *args[] = {&v, &L, &R, &tp, &plim};
                        rc = B.add(B.g, &prev, f, ns_cla_grid(I, f, smem, ns_pat, tp, L.n), smem, args);
                    }
                    int first = I->kpad / kTcM;
                    int nt = I->npat_pad / kTcM - first;
                    if (!rc && tc && nt > 0) {
                        size_t tsm = 0;
                        void *prep = nullptr;
                        void *f = tc_func(I->S, I->R, &tsm, &prep);
                        unsigned char *tab = I->d_tctab;
                        void *pargs[] = {&v, &L, &tab};
                        rc = B.add(B.g, &prev, prep, dim3(L.n), 0, pargs);
                        void *args[] = {&v, &L, &first, &nt, &tab};
                        B.block = dim3(kTcThreads);
                        if (!rc) rc = B.add(B.g, &prev, f, tc_grid(I, nt, L.n), tsm, args);
                        B.block = dim3(kThreads);
                    }
                }
                if (rc) return rc;
            }
        }
        // Newton loop of this branch: WHILE(not converged) { one iteration }
        NrSlot *slot = I->d_slots + nb.transMatIndex;
        int mat = nb.transMatIndex;
        cudaGraphConditionalHandle h;
        GB_CUDA(cudaGraphConditionalHandleCreate(&h, B.g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cn;
        GB_CUDA(cudaGraphAddNode(&cn, B.g, prev ? &prev : nullptr, prev ? 1 : 0, &cp));
        prev = cn;
        B.nodes++;
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaGraphNode_t bprev = nullptr;
        int pb = nb.partialIndex - I->ntip;
        int tip = nb.childIndex < I->ntip;
        int cb = tip ? nb.childIndex : nb.childIndex - I->ntip;
        if (dna) {
            long long es = I->eig_stride();
            void *args[] = {&v, &slot, &pb, &cb, &mat, &tip, &prm, &I->d_len, &I->d_eigen, &es, &I->d_rates, &h};
            rc = B.add(body, &bprev, nr_iter4_func(I->R, garli), dim3(nblocks), pmat_smem, args);
            if (rc) return rc;
        } else {
            int ws = 0;
            {
                int R = I->R, tp = ns_edge_tp;
                void *args[] = {&v, &pb, &cb, &mat, &tip, &ws, &R, &tp};
                rc = B.add(body, &bprev, ns_edge_func(I->S, garli, true), dim3(nblocks), ns_edge_smem, args);
                if (rc) return rc;
            }
            {
                int nbk = nblocks;
                void *args[] = {&slot, &I->d_block_sums, &nbk, &I->d_len, &mat, &prm, &h};
                rc = B.add(body, &bprev, (void *)k_nr_decide, dim3(1), 0, args);
                if (rc) return rc;
            }
            {
                long long es = I->eig_stride(), ms = I->mat_stride();
                int S = I->S, R = I->R, hp = I->has_pinv, e0 = 0;
                double pinv = I->pinv;
                void *args[] = {&I->d_eigen, &es, &S, &R, &I->d_rates, &pinv, &hp, &mat, &e0, &I->d_len, &I->d_mats, &ms};
                rc = B.add(body, &bprev, (void *)k_pmat_len, dim3(pmat_chunks(I->S, I->R)), pmat_smem, args);
                if (rc) return rc;
            }
        }
    }
    cudaError_t e = cudaGraphInstantiate(&I->graph_exec, B.g, 0);
    if (e != cudaSuccess) {
        g_last_error = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
        return GB_ERROR_GENERAL;
    }
    I->graph_nodes = B.nodes;
    return GB_SUCCESS;
}

// Enqueue the pass as one cooperative launch of k_pass4 (4-state data).
static int launch_persistent_pass(Instance *I, const gb_nr_branch *br, int nbr,
                                  const std::vector<std::vector<std::vector<DevOp>>> &levels, int rescaleEvery,
                                  NrParams prm, unsigned long long key) {
    std::vector<PCmd> cmds;
    std::vector<DevOp> flat;
    for (int b = 0; b < nbr; b++) {
        for (auto &lv : levels[b]) {
            PCmd c;
            c.type = kCmdLevel;
            c.a = (int)flat.size();
            c.b = (int)lv.size();
            c.c = c.d = 0;
            flat.insert(flat.end(), lv.begin(), lv.end());
            cmds.push_back(c);
        }
        PCmd c;
        c.type = kCmdNewton;
        c.a = br[b].partialIndex - I->ntip;
        const int tip = br[b].childIndex < I->ntip;
        c.b = tip ? br[b].childIndex : br[b].childIndex - I->ntip;
        c.c = tip;
        c.d = br[b].transMatIndex;
        cmds.push_back(c);
    }
    if (cmds.size() > I->cap_cmds) {
        if (I->d_cmds) cudaFree(I->d_cmds);
        I->cap_cmds = cmds.size() * 2;
        GB_CUDA(cudaMalloc(&I->d_cmds, I->cap_cmds * sizeof(PCmd)));
        I->pass_key = 0;
    }
    if (flat.size() > I->cap_pops || !I->d_pops) {
        if (I->d_pops) cudaFree(I->d_pops);
        I->cap_pops = std::max<size_t>(16, flat.size() * 2);
        GB_CUDA(cudaMalloc(&I->d_pops, I->cap_pops * sizeof(DevOp)));
        I->pass_key = 0;
    }
    if (key != I->pass_key) {
        GB_CUDA(cudaMemcpyAsync(I->d_cmds, cmds.data(), cmds.size() * sizeof(PCmd), cudaMemcpyHostToDevice, I->stream));
        if (!flat.empty())
            GB_CUDA(cudaMemcpyAsync(I->d_pops, flat.data(), flat.size() * sizeof(DevOp), cudaMemcpyHostToDevice, I->stream));
        I->pass_key = key;
    }
    GB_CUDA(cudaMemsetAsync(I->d_gsync, 0, sizeof(GridSync), I->stream));
    View v = make_view(I);
    v.rescale_every = rescaleEvery;
    PassArgs A;
    A.cmds = I->d_cmds;
    A.ncmd = (int)cmds.size();
    A.ops = I->d_pops;
    A.prm = prm;
    A.lengths = I->d_len;
    A.eig = I->d_eigen;
    A.rates = I->d_rates;
    A.slots = I->d_slots;
    A.gs = I->d_gsync;
    A.sums2 = I->d_sums2;
    A.nvb = I->nvb4;
    A.trace = I->d_trace;
    A.trace_cap = I->trace_cap;
    void *func = pass4_func(I->R, !I->mixed);
    int per_sm = 0;
    GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, kThreads, 0));
    if (per_sm < 1) {
        g_last_error = "persistent pass kernel cannot be resident";
        return GB_ERROR_NO_RESOURCE;
    }
    dim3 grid(std::min(per_sm * I->nsm, I->nvb4));
    void *args[] = {&v, &A};
    GB_CUDA(cudaLaunchCooperativeKernel(func, grid, dim3(kThreads), args, 0, I->stream));
    I->launches += 1;
    return GB_SUCCESS;
}

}  // namespace gb

extern "C" {

int gb_set_branch_lengths(int instance, const double *lengths, int count) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (count < 0 || count > I->nmat) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(I->d_len, lengths, count * sizeof(double), cudaMemcpyHostToDevice, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_get_branch_lengths(int instance, double *lengths, int count) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (count < 0 || count > I->nmat) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpyAsync(lengths, I->d_len, count * sizeof(double), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    return GB_SUCCESS;
}

int gb_newton_pass(int instance, const gb_nr_branch *branches, int branchCount, const gb_cla_operation *ops,
                   int opCount, int rescaleEvery, double precision, double minLength, double maxLength,
                   double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (branchCount < 0 || opCount < 0 || !(precision > 0.0) || !(minLength > 0.0) || !(maxLength > minLength))
        return GB_ERROR_OUT_OF_RANGE;
    for (int b = 0; b < branchCount; b++) {
        const gb_nr_branch &nb = branches[b];
        if (nb.transMatIndex < 0 || nb.transMatIndex >= I->nmat || nb.firstOp < 0 || nb.opCount < 0 ||
            nb.firstOp + nb.opCount > opCount || nb.partialIndex < I->ntip ||
            nb.partialIndex >= I->ntip + I->nbuf || nb.childIndex < 0 || nb.childIndex >= I->ntip + I->nbuf)
            return GB_ERROR_OUT_OF_RANGE;
    }
    cudaSetDevice(I->device);
    NrParams prm{precision, minLength, maxLength};
    // prepare every branch's CLA updates (this applies the rank rule, as executing them would)
    const std::vector<int> rank_before = I->rank;
    std::vector<std::vector<std::vector<DevOp>>> levels(branchCount);
    unsigned long long key = 1469598103934665603ULL;
    for (int b = 0; b < branchCount; b++) {
        int rc = prepare_ops(I, ops + branches[b].firstOp, branches[b].opCount, rescaleEvery, levels[b]);
        if (rc) {
            I->rank = rank_before;
            return rc;
        }
        for (auto &lv : levels[b]) key = fnv(key, lv.data(), sizeof(DevOp) * lv.size());
        key = fnv(key, &branches[b], sizeof(gb_nr_branch));
    }
    key = fnv(key, &rescaleEvery, sizeof(int));
    key = fnv(key, &prm, sizeof(prm));
    key = fnv(key, &I->version, sizeof(I->version));
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, I->device);
    const bool persistent = I->S == 4 && I->use_persistent && coop;
    if (persistent) {
        int rc = launch_persistent_pass(I, branches, branchCount, levels, rescaleEvery, prm, key);
        if (rc) {
            I->rank = rank_before;
            return rc;
        }
    } else if (key != I->graph_key || !I->graph_exec) {
        int rc = build_pass_graph(I, branches, branchCount, levels, rescaleEvery, prm);
        if (rc) {
            I->rank = rank_before;
            I->graph_key = 0;
            return rc;
        }
        I->graph_key = key;
    }
    if (!persistent) {
        GB_CUDA(cudaGraphLaunch(I->graph_exec, I->stream));
        I->launches += I->graph_nodes;
    }
    std::vector<NrSlot> slots(I->nmat);
    GB_CUDA(cudaMemcpyAsync(slots.data(), I->d_slots, I->nmat * sizeof(NrSlot), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaMemcpyAsync(I->h_status, I->d_status, sizeof(int), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    double improve = 0.0, last = 0.0;
    long long evals = 0;
    for (int b = 0; b < branchCount; b++) {
        const NrSlot &sl = slots[branches[b].transMatIndex];
        improve += sl.st.totalEstImprove;
        evals += sl.evals;
        last = sl.lnL;
    }
    if (out) {
        out[0] = improve;
        out[1] = last;
        out[2] = (double)evals;
    }
    I->site_valid = true;
    I->site_deriv_valid = false;
    if (*I->h_status & kStatusBarrierTimeout) {
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        g_last_error = "persistent pass: grid barrier wait exceeded its bound";
        return GB_ERROR_GENERAL;
    }
    if (*I->h_status & kStatusRescaleRetry) {
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
        I->graph_key = 0;
        return GB_ERROR_RESCALE_RETRY;
    }
    return GB_SUCCESS;
}

// Instrumentation: record up to `capacity` phase timestamps of the persistent
// pass kernel (block 0); capacity 0 switches it off.
int gb_set_pass_trace(int instance, int capacity) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    cudaSetDevice(I->device);
    if (I->d_trace) cudaFree(I->d_trace);
    I->d_trace = nullptr;
    I->trace_cap = 0;
    if (capacity > 0) {
        GB_CUDA(cudaMalloc(&I->d_trace, (size_t)capacity * sizeof(unsigned long long)));
        GB_CUDA(cudaMemset(I->d_trace, 0, (size_t)capacity * sizeof(unsigned long long)));
        I->trace_cap = capacity;
    }
    return GB_SUCCESS;
}

int gb_get_pass_trace(int instance, unsigned long long *out, int count) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!I->d_trace || count > I->trace_cap) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    GB_CUDA(cudaMemcpy(out, I->d_trace, (size_t)count * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    return GB_SUCCESS;
}

// 1 (default): 4-state passes run as one cooperative persistent kernel;
// 0: as a CUDA graph with a conditional WHILE node per branch
int gb_set_pass_mode(int instance, int persistent) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->use_persistent = persistent != 0;
    return GB_SUCCESS;
}

int gb_get_newton_state(int instance, int matrixIndex, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (matrixIndex < 0 || matrixIndex >= I->nmat) return GB_ERROR_OUT_OF_RANGE;
    cudaSetDevice(I->device);
    NrSlot sl;
    GB_CUDA(cudaMemcpyAsync(&sl, I->d_slots + matrixIndex, sizeof(NrSlot), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    out[0] = sl.st.v;
    out[1] = sl.st.totalEstImprove;
    out[2] = sl.lnL;
    out[3] = sl.d1;
    out[4] = sl.d2;
    out[5] = sl.evals;
    return GB_SUCCESS;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched candidate pass (gb_batch_newton): the host builds the command queue
// of k_batch4 (gb_batch.cuh) -- dependency levels of every candidate's CLA
// updates, then per step the step's CLA updates and one lockstep Newton
// command over all candidates, then a final score -- uploads it when it
// changes, and launches it cooperatively (captured once in a CUDA graph).
// ---------------------------------------------------------------------------
namespace gb {

// the plain form's batched pass (the precision form runs k_batch4m)
static void *batch4_func(int R) {
#define GB_CASE(r) \
    case r: return (void *)k_batch4<r, true>;
    switch (R) {
        GB_CASE(1) GB_CASE(2) GB_CASE(3) GB_CASE(4) GB_CASE(5) GB_CASE(6) GB_CASE(7) default : GB_CASE(8)
    }
#undef GB_CASE
}

template <typename T>
static int grow_device(T **p, size_t *cap, size_t need) {
    if (*p && need <= *cap) return GB_SUCCESS;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    const size_t c = std::max<size_t>(16, need + need / 2);
    GB_CUDA(cudaMalloc((void **)p, c * sizeof(T)));
    *cap = c;
    return GB_SUCCESS;
}

struct BatchPlan {
    std::vector<BCmd> cmds;
    std::vector<DevOp> ops;
    std::vector<BEntry> entries;    // plain form
    std::vector<MEntry> mentries;   // precision form
    int max_entries = 0;
    unsigned long long key = 0;
};

static void *batch4m_func(int R) {
    switch (R) {
        case 1: return (void *)k_batch4m<1>;
        case 2: return (void *)k_batch4m<2>;
        case 3: return (void *)k_batch4m<3>;
        case 4: return (void *)k_batch4m<4>;
        case 5: return (void *)k_batch4m<5>;
        case 6: return (void *)k_batch4m<6>;
        case 7: return (void *)k_batch4m<7>;
        default: return (void *)k_batch4m<8>;
    }
}

static void *coef4m_func(int R) {
    switch (R) {
        case 1: return (void *)k_coef4m<1>;
        case 2: return (void *)k_coef4m<2>;
        case 3: return (void *)k_coef4m<3>;
        case 4: return (void *)k_coef4m<4>;
        case 5: return (void *)k_coef4m<5>;
        case 6: return (void *)k_coef4m<6>;
        case 7: return (void *)k_coef4m<7>;
        default: return (void *)k_coef4m<8>;
    }
}

static void *level4m_func(int R) {
    switch (R) {
        case 1: return (void *)k_level4m<1>;
        case 2: return (void *)k_level4m<2>;
        case 3: return (void *)k_level4m<3>;
        case 4: return (void *)k_level4m<4>;
        case 5: return (void *)k_level4m<5>;
        case 6: return (void *)k_level4m<6>;
        case 7: return (void *)k_level4m<7>;
        default: return (void *)k_level4m<8>;
    }
}

// Enqueue one batched pass on the instance stream (no synchronisation).  The
// precision form runs its leading CLA levels as k_level4m launches, each
// coefficient pass as a k_coef4m launch, and every run of Newton / score
// commands between them in the persistent kernel.
static int enqueue_batch(Instance *I, const BatchPlan &P, NrParams prm, int rescaleEvery, int tiles, int chunks,
                         bool use_graph) {
    void *func = I->mixed ? batch4m_func(I->R) : batch4_func(I->R);
    int nlev = 0;
    if (I->mixed)
        while (nlev < (int)P.cmds.size() && P.cmds[nlev].type == kBLevel) nlev++;
    void *lfunc = I->mixed ? level4m_func(I->R) : nullptr;
    if (lfunc)
        GB_CUDA(cudaFuncSetAttribute(lfunc, cudaFuncAttributeMaxDynamicSharedMemorySize, cp_smem_bytes()));
    int per_sm = 0;
    GB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, kThreads, 0));
    if (per_sm < 1) {
        g_last_error = "batched pass kernel cannot be resident";
        return GB_ERROR_NO_RESOURCE;
    }
    View v = make_view(I);
    v.rescale_every = rescaleEvery;
    MixedArgs M;
    M.cmds = I->d_bcmds + nlev;
    M.ncmd = (int)P.cmds.size() - nlev;
    M.ops = I->d_bops;
    M.entries = I->d_mentries;
    M.slots = I->d_bslots;
    M.prm = prm;
    M.lengths = I->d_len;
    M.eig = I->d_eigen;
    M.rates = I->d_rates;
    M.coef = I->d_coef;
    M.cscale = I->d_cscale;
    M.etab = I->d_etab;
    M.chunk_sums = I->d_chunk_sums;
    M.active = I->d_active;
    M.nactive = I->d_active + 2 * P.max_entries;
    M.max_entries = P.max_entries;
    M.gs = I->d_gsync;
    M.tiles_per_item = tiles;
    M.chunks_per_item = chunks;
    M.trace = use_graph ? I->d_trace : nullptr;
    M.trace_cap = I->trace_cap;
    BatchArgs A;
    A.cmds = I->d_bcmds;
    A.ncmd = (int)P.cmds.size();
    A.ops = I->d_bops;
    A.entries = I->d_bentries;
    A.slots = I->d_bslots;
    A.prm = prm;
    A.lengths = I->d_len;
    A.eig = I->d_eigen;
    A.rates = I->d_rates;
    A.chunk_sums = I->d_chunk_sums;
    A.active = I->d_active;
    A.nactive = I->d_active + 2 * P.max_entries;
    A.max_entries = P.max_entries;
    A.gs = I->d_gsync;
    A.tiles_per_item = tiles;
    A.chunks_per_item = chunks;
    A.trace = use_graph ? I->d_trace : nullptr;
    A.trace_cap = I->trace_cap;
    void *args_plain[] = {&v, &A};
    void *args_mixed[] = {&v, &M};
    void **args = I->mixed ? args_mixed : args_plain;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(per_sm * I->nsm);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = I->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // the whole pass on the stream: level launches, then the persistent kernel
    // (none when the queue held levels only)
    const int G = I->R <= 1 ? 1 : I->R <= 2 ? 2 : I->R <= 4 ? 4 : 8;
    const int ctiles = (I->npat + kThreads / G - 1) / (kThreads / G);
    const int ncmd = (int)P.cmds.size();
    // phase timing: events around every launch, by phase (0 levels, 1 coefficient passes, 2 Newton / score)
    const bool timed = I->phase_timing && !use_graph;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pev;
    auto mark0 = [&](int phase) {
        if (!timed) return;
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, I->stream);
        pev.push_back({phase, {a, b}});
    };
    auto mark1 = [&]() {
        if (timed) cudaEventRecord(pev.back().second.second, I->stream);
    };
    auto launch_all = [&]() -> cudaError_t {
        cudaError_t e = cudaSuccess;
        for (int l = 0; l < nlev && e == cudaSuccess; l++) {
            const DevOp *ops = I->d_bops + P.cmds[l].a;
            int tpi = tiles;
            void *largs[] = {&v, (void *)&ops, &tpi};
            mark0(0);
            e = cudaLaunchKernel(lfunc, dim3((ctiles + tiles - 1) / tiles, P.cmds[l].b), dim3(kThreads), largs,
                                 cp_smem_bytes(), I->stream);
            mark1();
        }
        if (!I->mixed) {
            mark0(2);
            if (e == cudaSuccess) e = cudaMemsetAsync(I->d_gsync, 0, sizeof(GridSync), I->stream);
            if (e == cudaSuccess) e = cudaLaunchKernelExC(&cfg, func, args);
            mark1();
            return e;
        }
        for (int c = nlev; c < ncmd && e == cudaSuccess;) {
            if (P.cmds[c].type == kBCoef) {
                int first = P.cmds[c].a, tpi = tiles;
                void *cargs[] = {&v, &M, &first, &tpi};
                mark0(1);
                e = cudaLaunchKernel(coef4m_func(I->R), dim3((ctiles + tiles - 1) / tiles, P.cmds[c].b),
                                     dim3(kThreads), cargs, 0, I->stream);
                mark1();
                c++;
                continue;
            }
            int c1 = c;
            while (c1 < ncmd && P.cmds[c1].type != kBCoef) c1++;
            M.cmds = I->d_bcmds + c;
            M.ncmd = c1 - c;
            mark0(2);
            e = cudaMemsetAsync(I->d_gsync, 0, sizeof(GridSync), I->stream);
            if (e == cudaSuccess) e = cudaLaunchKernelExC(&cfg, func, args);
            mark1();
            c = c1;
        }
        return e;
    };
    auto resolve_phases = [&]() -> int {
        if (pev.empty()) return GB_SUCCESS;
        const cudaError_t se = cudaStreamSynchronize(I->stream);
        for (auto &x : pev) {
            float ms = 0.f;
            if (se == cudaSuccess && cudaEventElapsedTime(&ms, x.second.first, x.second.second) == cudaSuccess) {
                I->phase_ms[x.first] += ms;
                I->phase_launches[x.first]++;
            }
            cudaEventDestroy(x.second.first);
            cudaEventDestroy(x.second.second);
        }
        pev.clear();
        return se == cudaSuccess ? GB_SUCCESS : GB_ERROR_GENERAL;
    };
    int nkernels = nlev;
    for (int c = nlev; c < ncmd; c++)
        if (!I->mixed ? c == nlev : (P.cmds[c].type == kBCoef || c == nlev || P.cmds[c - 1].type == kBCoef))
            nkernels++;
    // the graph bakes in the work-item sizes, the rescale interval and the trace buffer: all of them key it
    unsigned long long gkey = P.key;
    const unsigned long long trace_ptr = reinterpret_cast<unsigned long long>(I->d_trace);
    gkey = fnv(gkey, &tiles, sizeof(tiles));
    gkey = fnv(gkey, &chunks, sizeof(chunks));
    gkey = fnv(gkey, &rescaleEvery, sizeof(rescaleEvery));
    gkey = fnv(gkey, &trace_ptr, sizeof(trace_ptr));
    if (use_graph && I->use_batch_graph && !I->phase_timing) {
        if (gkey != I->bgraph_key || !I->bgraph_exec) {
            if (I->bgraph_exec) cudaGraphExecDestroy(I->bgraph_exec);
            if (I->bgraph) cudaGraphDestroy(I->bgraph);
            I->bgraph_exec = nullptr;
            I->bgraph = nullptr;
            I->bgraph_key = 0;
            bool ok = cudaStreamBeginCapture(I->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
            if (ok) {
                const bool k = launch_all() == cudaSuccess;
                cudaGraph_t g = nullptr;
                const bool e = cudaStreamEndCapture(I->stream, &g) == cudaSuccess;
                ok = k && e && g;
                if (ok && cudaGraphInstantiate(&I->bgraph_exec, g, 0) != cudaSuccess) ok = false;
                if (ok) {
                    I->bgraph = g;
                    I->bgraph_key = gkey;
                } else {
                    if (g) cudaGraphDestroy(g);
                    I->bgraph_exec = nullptr;
                    I->use_batch_graph = 0;  // capture unsupported here: launch directly from now on
                }
            } else {
                I->use_batch_graph = 0;
            }
            cudaGetLastError();
        }
        if (I->bgraph_exec) {
            GB_CUDA(cudaGraphLaunch(I->bgraph_exec, I->stream));
            I->launches += nkernels;
            return GB_SUCCESS;
        }
    }
    const cudaError_t le = launch_all();
    const int prc = resolve_phases();
    GB_CUDA(le);
    I->launches += nkernels;
    return prc;
}

// Picks (CLA tiles, edge chunks) per work item by timing whole passes on the
// real batch.  Every trial starts from the same lengths and matrices (saved
// and restored on the device); the results do not depend on the choice.
static int autotune_batch(Instance *I, const BatchPlan &P, NrParams prm, int rescaleEvery) {
    struct PhaseOff {  // trial passes are not part of any phase measurement
        Instance *I;
        bool was;
        ~PhaseOff() { I->phase_timing = was; }
    } phase_off{I, I->phase_timing};
    I->phase_timing = false;
    const size_t len_bytes = (size_t)I->nmat * sizeof(double);
    const size_t mat_bytes = (size_t)I->nmat * I->mat_stride() * sizeof(double);
    double *save = nullptr;
    GB_CUDA(cudaMalloc((void **)&save, len_bytes + mat_bytes));
    GB_CUDA(cudaMemcpyAsync(save, I->d_len, len_bytes, cudaMemcpyDeviceToDevice, I->stream));
    GB_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(save) + len_bytes, I->d_mats, mat_bytes,
                            cudaMemcpyDeviceToDevice, I->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int tiles_plain[] = {1, 2, 4, 8}, tiles_mixed[] = {4, 8, 16, 32};
    const int *tiles_c = I->mixed ? tiles_mixed : tiles_plain;
    const int chunks_c[] = {1, 2, 4};
    float best = 1e30f;
    int bt = 1, bc = 1, rc = GB_SUCCESS;
    for (int ti = 0; ti < 4; ti++) {
        const int t = tiles_c[ti];
        for (int c : chunks_c) {
            for (int rep = 0; rep < 2 && rc == GB_SUCCESS; rep++) {  // first run warms up
                cudaMemcpyAsync(I->d_len, save, len_bytes, cudaMemcpyDeviceToDevice, I->stream);
                cudaMemcpyAsync(I->d_mats, reinterpret_cast<char *>(save) + len_bytes, mat_bytes,
                                cudaMemcpyDeviceToDevice, I->stream);
                cudaEventRecord(e0, I->stream);
                rc = enqueue_batch(I, P, prm, rescaleEvery, t, c, false);
                cudaEventRecord(e1, I->stream);
                if (cudaStreamSynchronize(I->stream) != cudaSuccess) rc = GB_ERROR_GENERAL;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep == 1 && ms < best) {
                    best = ms;
                    bt = t;
                    bc = c;
                }
            }
        }
    }
    cudaMemcpyAsync(I->d_len, save, len_bytes, cudaMemcpyDeviceToDevice, I->stream);
    cudaMemcpyAsync(I->d_mats, reinterpret_cast<char *>(save) + len_bytes, mat_bytes, cudaMemcpyDeviceToDevice,
                    I->stream);
    cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream);
    cudaStreamSynchronize(I->stream);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    if (rc) return rc;
    I->batch_tiles = bt;
    I->batch_chunks = bc;
    return GB_SUCCESS;
}

}  // namespace gb

extern "C" {

int gb_batch_newton(int instance, const gb_cla_operation *ops, int opCount, const gb_cla_operation *stepOps,
                    int stepOpCount, const gb_batch_step *steps, int candidateCount, int stepsPerCandidate,
                    int rescaleEvery, double precision, double minLength, double maxLength, double *out) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (I->S != 4) {
        g_last_error = "gb_batch_newton: 4-state data only";
        return GB_ERROR_NO_IMPLEMENTATION;
    }
    if (opCount < 0 || stepOpCount < 0 || candidateCount < 0 || stepsPerCandidate < 1 || !(precision > 0.0) ||
        !(minLength > 0.0) || !(maxLength > minLength) || (candidateCount > 0 && (!steps || !out)))
        return GB_ERROR_OUT_OF_RANGE;
    const int nC = candidateCount, K = stepsPerCandidate;
    for (int i = 0; i < nC * K; i++) {
        const gb_batch_step &s = steps[i];
        if (s.claOp < -1 || s.claOp >= stepOpCount || s.transMatIndex < 0 || s.transMatIndex >= I->nmat ||
            s.partialIndex < I->ntip || s.partialIndex >= I->ntip + I->nbuf || s.childIndex < 0 ||
            s.childIndex >= I->ntip + I->nbuf)
            return GB_ERROR_OUT_OF_RANGE;
    }
    cudaSetDevice(I->device);
    const std::vector<int> rank_before = I->rank;
    BatchPlan P;
    std::vector<std::vector<DevOp>> levels;
    int rc = prepare_ops(I, ops, opCount, rescaleEvery, levels, I->mixed);
    unsigned long long key = 1469598103934665603ULL;
    auto add_level = [&](const std::vector<DevOp> &lv) {
        BCmd c;
        c.type = kBLevel;
        c.a = (int)P.ops.size();
        c.b = (int)lv.size();
        P.ops.insert(P.ops.end(), lv.begin(), lv.end());
        P.cmds.push_back(c);
    };
    if (rc == GB_SUCCESS)
        for (auto &lv : levels) add_level(lv);
    for (int k = 0; k < K && rc == GB_SUCCESS && I->mixed && nC > 0; k++) {
        // precision form: the step's partial is formed inside the coefficient pass
        BCmd cc;
        cc.type = kBCoef;
        cc.a = (int)P.mentries.size();
        cc.b = nC;
        auto side = [&](int b, int &idx, int &tip) {
            tip = b < I->ntip;
            idx = tip ? b : b - I->ntip;
        };
        auto is_wide = [&](int idx, int tip) { return !tip && idx >= 0 && I->wide[idx] == 1; };
        for (int c = 0; c < nC; c++) {
            const gb_batch_step &s = steps[c * K + k];
            MEntry m;
            if (s.claOp >= 0) {
                const gb_cla_operation &o = stepOps[s.claOp];
                if (o.childClaIndex1 < 0 || o.childClaIndex1 >= I->ntip + I->nbuf || o.childClaIndex2 < 0 ||
                    o.childClaIndex2 >= I->ntip + I->nbuf || o.transMatIndex1 < 0 || o.transMatIndex1 >= I->nmat ||
                    o.transMatIndex2 < 0 || o.transMatIndex2 >= I->nmat)
                    rc = GB_ERROR_OUT_OF_RANGE;
                side(o.childClaIndex1, m.b1, m.t1);
                side(o.childClaIndex2, m.b2, m.t2);
                m.m1 = o.transMatIndex1;
                m.m2 = o.transMatIndex2;
            } else {
                side(s.partialIndex, m.b1, m.t1);
                m.m1 = -1;
                m.b2 = -1;
                m.t2 = 0;
                m.m2 = -1;
            }
            side(s.childIndex, m.bk, m.tk);
            m.mk = s.transMatIndex;
            m.wide = (is_wide(m.b1, m.t1) ? 1 : 0) | (is_wide(m.b2, m.t2) ? 2 : 0) | (is_wide(m.bk, m.tk) ? 4 : 0);
            if ((m.b1 >= 0 && !m.t1 && I->wide[m.b1] == 2) || (m.b2 >= 0 && !m.t2 && I->wide[m.b2] == 2) ||
                (!m.tk && I->wide[m.bk] == 2))
                rc = GB_ERROR_OUT_OF_RANGE;
            P.mentries.push_back(m);
        }
        P.cmds.push_back(cc);
        BCmd nc = cc;
        nc.type = kBNewton;
        P.cmds.push_back(nc);
    }
    for (int k = 0; k < K && rc == GB_SUCCESS && !I->mixed && nC > 0; k++) {
        std::vector<gb_cla_operation> sops;
        for (int c = 0; c < nC; c++)
            if (steps[c * K + k].claOp >= 0) {
                gb_cla_operation o = stepOps[steps[c * K + k].claOp];
                o.opDepLevel = 1;  // the ops of one step are independent of each other
                sops.push_back(o);
            }
        std::vector<std::vector<DevOp>> sl;
        rc = prepare_ops(I, sops.data(), (int)sops.size(), rescaleEvery, sl, false);
        if (rc) break;
        for (auto &lv : sl) add_level(lv);
        BCmd nc;
        nc.type = kBNewton;
        nc.a = (int)P.entries.size();
        nc.b = nC;
        for (int c = 0; c < nC; c++) {
            const gb_batch_step &s = steps[c * K + k];
            BEntry e;
            e.pbuf = s.partialIndex - I->ntip;
            e.tip = s.childIndex < I->ntip;
            e.cbuf = e.tip ? s.childIndex : s.childIndex - I->ntip;
            e.mat = s.transMatIndex;
            P.entries.push_back(e);
        }
        P.cmds.push_back(nc);
    }
    if (rc) {
        I->rank = rank_before;
        return rc;
    }
    if (nC > 0) {
        BCmd fs;  // lnL of every candidate at its optimised lengths
        fs.type = kBScore;
        fs.a = (K - 1) * nC;
        fs.b = nC;
        P.cmds.push_back(fs);
    }
    P.max_entries = nC;
    // key of the captured graph: what its launches take as arguments -- the
    // command list (level and entry counts, offsets), the candidate count, the
    // Newton parameters and the instance's data version; the ops and entries
    // themselves are read from device memory, uploaded on every call
    const double nrp[3] = {precision, minLength, maxLength};
    key = fnv(key, P.cmds.data(), sizeof(BCmd) * P.cmds.size());
    key = fnv(key, &nC, sizeof(nC));
    key = fnv(key, nrp, sizeof(nrp));
    key = fnv(key, &I->version, sizeof(I->version));
    P.key = key;
    const int nchunks = (I->npat + kChunk - 1) / kChunk;
    const size_t nent = I->mixed ? P.mentries.size() : P.entries.size();
    bool realloc = false;
    {
        const void *before[] = {I->d_bcmds, I->d_bops, I->d_bentries, I->d_bslots, I->d_chunk_sums, I->d_active,
                                I->d_mentries, I->d_coef, I->d_cscale, I->d_etab};
        if (I->mixed &&
            ((rc = grow_device(&I->d_mentries, &I->cap_mentries, nent)) ||
             (rc = grow_device(&I->d_coef, &I->cap_coef, (size_t)nC * (1 + 3 * I->R) * I->npat_pad)) ||
             (rc = grow_device(&I->d_cscale, &I->cap_cscale, (size_t)nC * I->npat_pad)) ||
             (rc = grow_device(&I->d_etab, &I->cap_etab, (size_t)nC * 3 * (1 + 3 * I->R))))) {
            I->rank = rank_before;
            return rc;
        }
        if ((rc = grow_device(&I->d_bcmds, &I->cap_bcmds, P.cmds.size())) ||
            (rc = grow_device(&I->d_bops, &I->cap_bops, std::max<size_t>(1, P.ops.size()))) ||
            (rc = grow_device(&I->d_bentries, &I->cap_bentries, std::max<size_t>(1, P.entries.size()))) ||
            (rc = grow_device(&I->d_bslots, &I->cap_bslots, nent)) ||
            (rc = grow_device(&I->d_chunk_sums, &I->cap_chunk, (size_t)nC * nchunks * 3)) ||
            (rc = grow_device(&I->d_active, &I->cap_active, (size_t)2 * nC + 2))) {
            I->rank = rank_before;
            return rc;
        }
        const void *after[] = {I->d_bcmds, I->d_bops, I->d_bentries, I->d_bslots, I->d_chunk_sums, I->d_active,
                               I->d_mentries, I->d_coef, I->d_cscale, I->d_etab};
        for (int i = 0; i < 10; i++) realloc = realloc || before[i] != after[i];
    }
    if (realloc) I->bgraph_key = 0;
    GB_CUDA(cudaMemcpyAsync(I->d_bcmds, P.cmds.data(), P.cmds.size() * sizeof(BCmd), cudaMemcpyHostToDevice,
                            I->stream));
    if (!P.ops.empty())
        GB_CUDA(cudaMemcpyAsync(I->d_bops, P.ops.data(), P.ops.size() * sizeof(DevOp), cudaMemcpyHostToDevice,
                                I->stream));
    if (!P.entries.empty())
        GB_CUDA(cudaMemcpyAsync(I->d_bentries, P.entries.data(), P.entries.size() * sizeof(BEntry),
                                cudaMemcpyHostToDevice, I->stream));
    if (!P.mentries.empty())
        GB_CUDA(cudaMemcpyAsync(I->d_mentries, P.mentries.data(), P.mentries.size() * sizeof(MEntry),
                                cudaMemcpyHostToDevice, I->stream));
    NrParams prm{precision, minLength, maxLength};
    int tiles = I->batch_tiles, chunks = I->batch_chunks;
    if (tiles == 0 || chunks == 0) {
        if (nC > 0) {
            if ((rc = autotune_batch(I, P, prm, rescaleEvery))) {
                I->rank = rank_before;
                return rc;
            }
            tiles = I->batch_tiles;
            chunks = I->batch_chunks;
        } else {  // levels only (a base tree): not worth tuning for
            tiles = I->mixed ? 16 : 4;
            chunks = 1;
        }
    }
    cudaEvent_t te0 = nullptr, te1 = nullptr;
    if (I->timing && nC > 0) {
        cudaEventCreate(&te0);
        cudaEventCreate(&te1);
        cudaEventRecord(te0, I->stream);
    }
    if ((rc = enqueue_batch(I, P, prm, rescaleEvery, tiles, chunks, nC > 0 && !I->phase_timing))) {
        I->rank = rank_before;
        return rc;
    }
    if (te1) cudaEventRecord(te1, I->stream);
    std::vector<BSlot> slots(nent);
    GB_CUDA(cudaMemcpyAsync(slots.data(), I->d_bslots, slots.size() * sizeof(BSlot), cudaMemcpyDeviceToHost,
                            I->stream));
    GB_CUDA(cudaMemcpyAsync(I->h_status, I->d_status, sizeof(int), cudaMemcpyDeviceToHost, I->stream));
    GB_CUDA(cudaStreamSynchronize(I->stream));
    if (te1) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, te0, te1);
        I->batch_ms += ms;
        I->batch_timed++;
        cudaEventDestroy(te0);
        cudaEventDestroy(te1);
    }
    for (int c = 0; c < nC; c++) {
        double imp = 0.0;
        long long ev = 0;
        for (int k = 0; k < K; k++) {
            imp += slots[k * nC + c].st.totalEstImprove;
            ev += slots[k * nC + c].evals;
        }
        out[4 * c] = slots[c].first_lnL;
        out[4 * c + 1] = slots[(K - 1) * nC + c].score;
        out[4 * c + 2] = imp;
        out[4 * c + 3] = (double)ev;
    }
    const int st = *I->h_status;
    if (st) {
        GB_CUDA(cudaMemsetAsync(I->d_status, 0, sizeof(int), I->stream));
        GB_CUDA(cudaStreamSynchronize(I->stream));
    }
    if (st & kStatusBarrierTimeout) {
        g_last_error = "batched pass: grid barrier wait exceeded its bound";
        return GB_ERROR_GENERAL;
    }
    if (st & kStatusRescaleRetry) return GB_ERROR_RESCALE_RETRY;
    return GB_SUCCESS;
}

// Work-item sizes of the batched pass: CLA tiles (64 patterns at 4 categories)
// and edge chunks (256 patterns) per work item; 0, 0 = autotune on the next call.
int gb_set_batch_tuning(int instance, int tilesPerItem, int chunksPerItem) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (tilesPerItem < 0 || tilesPerItem > 64 || chunksPerItem < 0 || chunksPerItem > 64) return GB_ERROR_OUT_OF_RANGE;
    I->batch_tiles = tilesPerItem;
    I->batch_chunks = chunksPerItem;
    I->bgraph_key = 0;
    return GB_SUCCESS;
}

int gb_set_eigen_from_rate_matrices(int instance, int count, const int *eigenIndices, const double *Q,
                                    const double *pi, const double *blenMults, int *sweepsOut) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (count < 1 || !eigenIndices || !Q || !pi || !blenMults) return GB_ERROR_OUT_OF_RANGE;
    const int S = I->S;
    for (int c = 0; c < count; c++) {
        if (eigenIndices[c] < 0 || eigenIndices[c] >= I->neigen) return GB_ERROR_OUT_OF_RANGE;
        for (int i = 0; i < S; i++)
            if (!(pi[c * S + i] > 0.0)) return GB_ERROR_OUT_OF_RANGE;  // D^1/2 needs positive frequencies
    }
    cudaSetDevice(I->device);
    if (count > I->cap_eig) {
        // the previous scratch may still be read by queued work
        GB_CUDA(cudaStreamSynchronize(I->stream));
        cudaFree(I->d_eq);
        cudaFree(I->d_epi);
        cudaFree(I->d_ejobs);
        cudaFree(I->d_esw);
        I->d_eq = I->d_epi = nullptr;
        I->d_ejobs = nullptr;
        I->d_esw = nullptr;
        I->cap_eig = 0;
        if (cudaMalloc(&I->d_eq, (size_t)count * S * S * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&I->d_epi, (size_t)count * S * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&I->d_ejobs, (size_t)count * sizeof(EigenJob)) != cudaSuccess ||
            cudaMalloc(&I->d_esw, (size_t)count * sizeof(int)) != cudaSuccess) {
            g_last_error = "gb_set_eigen_from_rate_matrices: cudaMalloc failed";
            return GB_ERROR_OUT_OF_MEMORY;
        }
        I->cap_eig = count;
    }
    double *dQ = I->d_eq, *dpi = I->d_epi;
    EigenJob *djobs = I->d_ejobs;
    int *dsw = I->d_esw;
    std::vector<EigenJob> jobs(count);
    for (int c = 0; c < count; c++) {
        jobs[c].Q = dQ + (size_t)c * S * S;
        jobs[c].pi = dpi + (size_t)c * S;
        jobs[c].blen_mult = blenMults[c];
        jobs[c].out = I->d_eigen + (size_t)eigenIndices[c] * I->eig_stride();
        jobs[c].sweeps = dsw + c;
    }
    int rc = GB_SUCCESS;
    if (cudaMemcpyAsync(dQ, Q, (size_t)count * S * S * sizeof(double), cudaMemcpyHostToDevice, I->stream) ||
        cudaMemcpyAsync(dpi, pi, (size_t)count * S * sizeof(double), cudaMemcpyHostToDevice, I->stream) ||
        cudaMemcpyAsync(djobs, jobs.data(), (size_t)count * sizeof(EigenJob), cudaMemcpyHostToDevice, I->stream))
        rc = GB_ERROR_GENERAL;
    if (!rc) {
        k_eigen_jacobi<<<count, 256, eigen_smem_bytes(S), I->stream>>>(djobs, S);
        rc = check_launch(I);
    }
    std::vector<int> sw(count, 0);
    if (!rc && cudaMemcpyAsync(sw.data(), dsw, (size_t)count * sizeof(int), cudaMemcpyDeviceToHost, I->stream))
        rc = GB_ERROR_GENERAL;
    if (cudaStreamSynchronize(I->stream) != cudaSuccess) rc = GB_ERROR_GENERAL;
    if (rc) return rc;
    if (sweepsOut)
        for (int c = 0; c < count; c++) sweepsOut[c] = sw[c];
    for (int c = 0; c < count; c++)
        if (sw[c] >= kJacobiMaxSweeps) {
            g_last_error = "gb_set_eigen_from_rate_matrices: Jacobi iteration did not converge";
            return GB_ERROR_FLOATING_POINT;
        }
    I->version++;
    return GB_SUCCESS;
}

int gb_set_tensor_cores(int instance, int on) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->use_tc = on != 0;
    I->graph_key = 0;
    return GB_SUCCESS;
}

int gb_set_buffer_precision(int instance, int bufferIndex, int fp64) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!I->mixed) return GB_ERROR_NO_IMPLEMENTATION;  // the plain form is FP64 throughout
    const int b = bufferIndex - I->ntip;
    if (b < 0 || b + 1 >= I->nbuf) return GB_ERROR_OUT_OF_RANGE;
    if (fp64) {
        if (I->wide[b] == 2 || I->wide[b + 1] == 1) return GB_ERROR_OUT_OF_RANGE;
        I->wide[b] = 1;
        I->wide[b + 1] = 2;
    } else if (I->wide[b] == 1) {
        I->wide[b] = 0;
        I->wide[b + 1] = 0;
    }
    I->version++;
    return GB_SUCCESS;
}

int gb_get_batch_timing(int instance, double *out2) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out2[0] = I->batch_ms;
    out2[1] = (double)I->batch_timed;
    return GB_SUCCESS;
}

int gb_set_batch_phase_timing(int instance, int on) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    I->phase_timing = on != 0;
    return GB_SUCCESS;
}

int gb_get_batch_phase_timing(int instance, double *out6) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!out6) return GB_ERROR_OUT_OF_RANGE;
    for (int k = 0; k < 3; k++) {
        out6[2 * k] = I->phase_ms[k];
        out6[2 * k + 1] = (double)I->phase_launches[k];
    }
    return GB_SUCCESS;
}

int gb_get_batch_tuning(int instance, int *out3) {
    Instance *I = get(instance);
    if (!I) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out3[0] = I->batch_tiles;
    out3[1] = I->batch_chunks;
    out3[2] = I->use_batch_graph && I->bgraph_exec ? 1 : 0;
    return GB_SUCCESS;
}

}  // extern "C"
