// gb_newton_dna.cuh -- one fused Newton-Raphson iteration for 4-state data.
//
// All blocks evaluate lnL, d1 and d2 over their patterns exactly as k_edge4
// does (same grid, same per-block sums); the last block to finish reduces the
// partial sums in k_reduce3's order, takes gb::nr_step, writes the new branch
// length and recomputes P(t), dP/dt and d2P/dt2 at it (Model::CalcDerivatives,
// model.cpp:1271) -- one kernel per iteration instead of three.
#pragma once
#include "gb_dna.cuh"
#include "gb_graph.cuh"
#include "gb_pmat.cuh"

namespace gb {

template <int R, bool GARLI_SCALE>
__global__ void __launch_bounds__(kThreads) k_nr_iter4(View v, NrSlot *slot, int pbuf, int cbuf, int mat,
                                                        int child_tip, NrParams prm, double *lengths,
                                                        const double *eig, long long eig_stride,
                                                        const double *rates, cudaGraphConditionalHandle h) {
    __shared__ EdgeSmem<R, true> sm;
    __shared__ bool s_last;
    __shared__ double red[3][kThreads];
    edge4_load_smem<R, true>(v, mat, sm);
    __syncthreads();
    double accL = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < v.npat; p += gridDim.x * blockDim.x) {
        if (p < v.kpad)
            edge4_site<double, R, GARLI_SCALE, true>(v, sm, pbuf, cbuf, child_tip, 0, p, accL, acc1, acc2);
        else
            edge4_site<float, R, GARLI_SCALE, true>(v, sm, pbuf, cbuf, child_tip, 0, p, accL, acc1, acc2);
    }
    block_sum3(accL, acc1, acc2, v.block_sums + 3 * blockIdx.x);
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned ticket = atomicAdd(&slot->arrived, 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the reduction of k_reduce3, over this launch's nblocks partial sums
    {
        const volatile double *parts = v.block_sums;
        double a = 0.0, b = 0.0, c = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            a += parts[3 * i];
            b += parts[3 * i + 1];
            c += parts[3 * i + 2];
        }
        red[0][threadIdx.x] = a;
        red[1][threadIdx.x] = b;
        red[2][threadIdx.x] = c;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) {
                red[0][threadIdx.x] += red[0][threadIdx.x + w];
                red[1][threadIdx.x] += red[1][threadIdx.x + w];
                red[2][threadIdx.x] += red[2][threadIdx.x + w];
            }
            __syncthreads();
        }
    }
    __shared__ double s_len;
    if (threadIdx.x == 0) {
        const double lnL = red[0][0], d1 = red[1][0], d2 = red[2][0];
        if (slot->evals == 0) nr_init(slot->st, lengths[mat], prm.min_brlen, prm.max_brlen);
        slot->lnL = lnL;
        slot->d1 = d1;
        slot->d2 = d2;
        slot->evals++;
        const int fin = nr_step(slot->st, d1, d2, lnL, prm.precision, prm.min_brlen, prm.max_brlen);
        lengths[mat] = slot->st.v;
        slot->arrived = 0;
        s_len = slot->st.v;
        cudaGraphSetConditional(h, fin ? 0u : 1u);
    }
    __syncthreads();
    // P(t), dP, d2P at the new length for the next iteration / the next branches
    TransOp op;
    op.dest = mat;
    op.eigen = 0;
    op.derivs = 1;
    op.t = s_len;
    pmat_body(eig, eig_stride, 4, R, rates, v.pinv, v.has_pinv, op, const_cast<double *>(v.mats), v.mat_stride, 0, 1);
}

}  // namespace gb
