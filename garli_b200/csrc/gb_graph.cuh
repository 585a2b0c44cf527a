// gb_graph.cuh -- device side of the graph-resident branch-optimisation pass.
//
// For every branch of OptimizeAllBranches (optimization.cpp:97, :1042) the
// pass graph holds the CLA updates the branch's derivatives need, then a
// conditional WHILE node whose body is one Newton-Raphson iteration:
//   edge kernel (lnL, d1, d2 partial sums) -> k_nr_decide (FP64 reduction +
//   gb::nr_step, new length written to the device length array, loop flag) ->
//   k_pmat_len (P, dP, d2P at the new length).
// No host round trip happens between iterations or branches.
#pragma once
#include "gb_common.cuh"
#include "gb_newton.h"

namespace gb {

struct NrParams {
    double precision, min_brlen, max_brlen;
};

struct NrSlot {
    NrState st;
    double lnL, d1, d2;
    int evals;
    unsigned int arrived;  // blocks of the current fused iteration that finished
};

// Start of a pass: every slot is re-initialised lazily by its first iteration.
__global__ void k_nr_reset(NrSlot *slots, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        slots[i].evals = 0;
        slots[i].arrived = 0;
        slots[i].st.done = 0;
    }
}

__global__ void k_nr_begin(NrSlot *slot, const double *lengths, int mat, NrParams prm,
                           cudaGraphConditionalHandle h) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        nr_init(slot->st, lengths[mat], prm.min_brlen, prm.max_brlen);
        slot->evals = 0;
        cudaGraphSetConditional(h, 1);
    }
}

// Reduces the edge kernel's per-block partial sums in exactly the order of
// k_reduce3 (so host- and device-driven passes see identical lnL/d1/d2), then
// takes one Newton step.
__global__ void __launch_bounds__(kThreads) k_nr_decide(NrSlot *slot, const double *parts, int nblocks,
                                                        double *lengths, int mat, NrParams prm,
                                                        cudaGraphConditionalHandle h) {
    __shared__ double s[3][kThreads];
    double a = 0.0, b = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a += parts[3 * i];
        b += parts[3 * i + 1];
        c += parts[3 * i + 2];
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
        const double lnL = s[0][0], d1 = s[1][0], d2 = s[2][0];
        if (slot->evals == 0) nr_init(slot->st, lengths[mat], prm.min_brlen, prm.max_brlen);
        slot->lnL = lnL;
        slot->d1 = d1;
        slot->d2 = d2;
        slot->evals++;
        const int fin = nr_step(slot->st, d1, d2, lnL, prm.precision, prm.min_brlen, prm.max_brlen);
        lengths[mat] = slot->st.v;
        cudaGraphSetConditional(h, fin ? 0u : 1u);
    }
}

}  // namespace gb
