// gb_pmat.cuh -- FP64 transition matrices and the final FP64 reduction.
#pragma once
#include "gb_common.cuh"

namespace gb {

constexpr int kMaxTransOps = 64;

struct TransOp {
    int dest;
    int eigen;
    int derivs;
    double t;
};
struct TransOps {
    int n;
    TransOp op[kMaxTransOps];
};

// P(t), dP/dt, d2P/dt2 for every rate category, one block per matrix:
//   Model::AltCalcPmat   model.cpp:1469-1597
//   Model::CalcDerivatives model.cpp:1271-1358
// scaledEigVal = lambda * rate [/(1-pinv)]; e_k = exp(scaledEigVal * t);
// P_ij = max(0, sum_k (U_ik Uinv_kj) e_k) with the k sum sequential.
// eig layout per eigen index: [lambda (S) | U (S*S) | Uinv (S*S)], lambda pre-scaled
// by the blen multiplier.
// outputs per block of one matrix: R*S*S split over pmat_chunks(S, R) blocks
__host__ __device__ constexpr int pmat_chunks(int S, int R) {
    return (R * S * S + 511) / 512 < 16 ? (R * S * S + 511) / 512 : 16;
}
// dynamic shared memory of a P(t) block: the exponential tables and, for 20
// and 61 states, U and U^-1 (read S times per output)
__host__ __device__ constexpr size_t pmat_smem_bytes(int S, int R) {
    return (3 * (size_t)R * S + (S > 4 ? 2 * (size_t)S * S : 0)) * sizeof(double);
}

__device__ __forceinline__ void pmat_body(const double *eig, long long eig_stride, int S, int R,
                                          const double *rates, double pinv, int has_pinv, const TransOp op,
                                          double *mats, long long mat_stride, int chunk, int nchunks) {
    extern __shared__ double sh[];
    double *ex = sh, *d1e = ex + R * S, *d2e = d1e + R * S;
    const double *lam = eig + (long long)op.eigen * eig_stride;
    const double *U = lam + S, *Ui = U + S * S;
    for (int idx = threadIdx.x; idx < R * S; idx += blockDim.x) {
        const int r = idx / S, k = idx % S;
        double sev = mul(lam[k], rates[r]);
        if (has_pinv) sev = sev / sub(1.0, pinv);
        const double e = exp(mul(sev, op.t));
        ex[idx] = e;
        d1e[idx] = mul(sev, e);
        d2e[idx] = mul(sev, d1e[idx]);
    }
    if (S > 4) {
        double *sU = d2e + R * S, *sUi = sU + S * S;
        for (int idx = threadIdx.x; idx < S * S; idx += blockDim.x) {
            sU[idx] = U[idx];
            sUi[idx] = Ui[idx];
        }
        U = sU;
        Ui = sUi;
    }
    __syncthreads();
    double *out = mats + (long long)op.dest * mat_stride;
    const int SS = S * S, n = R * SS, per = (n + nchunks - 1) / nchunks;
    const int i0 = chunk * per, i1 = min(n, i0 + per);
    for (int idx = i0 + threadIdx.x; idx < i1; idx += blockDim.x) {
        const int r = idx / SS, ij = idx % SS, i = ij / S, j = ij % S;
        const double *e = ex + r * S;
        double sp = 0.0, s1 = 0.0, s2 = 0.0;
        for (int k = 0; k < S; k++) {
            const double x = mul(U[i * S + k], Ui[k * S + j]);
            sp = add(sp, mul(x, e[k]));
            if (op.derivs) {
                s1 = add(s1, mul(x, d1e[r * S + k]));
                s2 = add(s2, mul(x, d2e[r * S + k]));
            }
        }
        out[idx] = sp > 0.0 ? sp : 0.0;
        if (op.derivs) {
            out[R * SS + idx] = s1;
            out[2 * R * SS + idx] = s2;
        }
    }
}

// Model slot table: per eigen index, [freqs (S) | category rates (R) |
// category weights (R) | pinv | has_pinv], model_slot_stride(S, R) doubles.
__host__ __device__ constexpr int model_slot_stride(int S, int R) { return S + 2 * R + 2; }

// grid (matrices, pmat_chunks(S, R)); each matrix takes the rates and pinv of
// its eigen index's model slot
__global__ void __launch_bounds__(kThreads) k_pmats(const double *eig, long long eig_stride, int S, int R,
                                                    const double *mslots, TransOps ops, double *mats,
                                                    long long mat_stride) {
    const TransOp op = ops.op[blockIdx.x];
    const double *slot = mslots + (long long)op.eigen * model_slot_stride(S, R);
    pmat_body(eig, eig_stride, S, R, slot + S, slot[S + 2 * R], slot[S + 2 * R + 1] != 0.0 ? 1 : 0, op, mats,
              mat_stride, blockIdx.y, gridDim.y);
}

// P(t), dP/dt, d2P/dt2 of one matrix whose branch length lives on the device
// (the Newton iterations of a device-side optimisation pass); grid pmat_chunks(S, R)
__global__ void __launch_bounds__(kThreads) k_pmat_len(const double *eig, long long eig_stride, int S, int R,
                                                       const double *rates, double pinv, int has_pinv, int dest,
                                                       int eigen, const double *lengths, double *mats,
                                                       long long mat_stride) {
    TransOp op;
    op.dest = dest;
    op.eigen = eigen;
    op.derivs = 1;
    op.t = lengths[dest];
    pmat_body(eig, eig_stride, S, R, rates, pinv, has_pinv, op, mats, mat_stride, blockIdx.x, gridDim.x);
}

// Sum the per-block partial sums of an edge evaluation (nblocks x 3) into
// out[0..2].  One block; each thread adds a fixed strided subset in order and
// the block combines them in a fixed tree, so the result is deterministic.
__global__ void __launch_bounds__(kThreads) k_reduce3(const double *parts, int nblocks, double *out) {
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
        out[0] = s[0][0];
        out[1] = s[1][0];
        out[2] = s[2][0];
    }
}

}  // namespace gb
