// gb_eigen.cuh -- FP64 eigen-decomposition of reversible rate matrices on the
// device, one CTA per model (Model::CalcEigenStuff, model.cpp:827-856).
//
// For a reversible Q (pi_i Q_ij = pi_j Q_ji), B = D^1/2 Q D^-1/2 with
// D = diag(pi) is symmetric, B = V diag(lambda) V^T with orthogonal V, and
// Q = U diag(lambda) U^-1 with U = D^-1/2 V, U^-1 = V^T D^1/2 -- the same
// eigensystem GARLI's EigenRealGeneral finds (up to order and the sign of
// each eigenvector, neither of which changes P(t)).  B is diagonalised by the
// cyclic Jacobi method with a round-robin ordering: each step rotates n/2
// disjoint (p, q) pairs at once (columns of A and V, then rows of A), a sweep
// is n - 1 steps; sweeps stop when the off-diagonal mass is below 1e-30 of the
// diagonal's, or after kJacobiMaxSweeps (a bound, never reached in practice:
// Jacobi converges quadratically).  The eigenvalues are stored multiplied by
// GARLI's blen_multiplier (model.cpp:845-846), in the engine's eigen layout
// [lambda | U | U^-1].
#pragma once
#include <cuda_runtime.h>

namespace gb {

constexpr int kEigenMaxN = 64;  // padded (even) dimension: up to 61 states
constexpr int kJacobiMaxSweeps = 40;

struct EigenJob {
    const double *Q;    // S x S row-major
    const double *pi;   // S
    double blen_mult;
    double *out;        // eigen slot: S eigenvalues, U (S x S), U^-1 (S x S)
    int *sweeps;        // sweeps used (diagnostic)
};

// Position of player j in round s of a round-robin over n players (player 0 fixed).
__device__ __forceinline__ int rr_pos(int j, int s, int n) { return j == 0 ? 0 : ((j - 1 + s) % (n - 1)) + 1; }

// dynamic shared memory: A and V, n x (n + 1) doubles each
__host__ __device__ constexpr size_t eigen_smem_bytes(int S) { return 2 * (size_t)((S + 1) & ~1) * (((S + 1) & ~1) + 1) * 8; }

__global__ void __launch_bounds__(256) k_eigen_jacobi(const EigenJob *jobs, int S) {
    extern __shared__ double esm[];
    __shared__ double sq[kEigenMaxN];
    __shared__ double rc[kEigenMaxN / 2], rs[kEigenMaxN / 2];
    __shared__ int rp[kEigenMaxN / 2], rq[kEigenMaxN / 2];
    __shared__ double red[2][256 / 32];
    __shared__ int s_done;
    const EigenJob job = jobs[blockIdx.x];
    const int n = (S + 1) & ~1;  // even: a zero row/column pads odd S
    const int np1 = n + 1;        // row pitch (odd: rows in different banks)
    double *Am = esm, *Vm = esm + n * np1;
#define A(i, j) Am[(i) * np1 + (j)]
#define V(i, j) Vm[(i) * np1 + (j)]
    const int t = threadIdx.x, nt = blockDim.x;
    for (int i = t; i < n; i += nt) sq[i] = i < S ? sqrt(job.pi[i]) : 1.0;
    __syncthreads();
    for (int idx = t; idx < n * n; idx += nt) {
        const int i = idx / n, j = idx % n;
        double b = 0.0;
        if (i < S && j < S) {
            // symmetrised exactly: the mean of the two mirrored entries
            const double bij = sq[i] * job.Q[i * S + j] / sq[j];
            const double bji = sq[j] * job.Q[j * S + i] / sq[i];
            b = 0.5 * (bij + bji);
        }
        A(i, j) = b;
        V(i, j) = i == j ? 1.0 : 0.0;
    }
    __syncthreads();
    int sweep = 0;
    for (; sweep < kJacobiMaxSweeps; sweep++) {
        // convergence: off-diagonal vs diagonal mass
        double off = 0.0, dia = 0.0;
        for (int idx = t; idx < n * n; idx += nt) {
            const int i = idx / n, j = idx % n;
            const double a = A(i, j);
            if (i == j) dia += a * a;
            else off += a * a;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            dia += __shfl_xor_sync(0xffffffffu, dia, o);
        }
        if ((t & 31) == 0) {
            red[0][t >> 5] = off;
            red[1][t >> 5] = dia;
        }
        __syncthreads();
        if (t == 0) {
            double o2 = 0.0, d2 = 0.0;
            for (int w = 0; w < nt / 32; w++) {
                o2 += red[0][w];
                d2 += red[1][w];
            }
            s_done = !(o2 > 1e-30 * d2);
        }
        __syncthreads();
        if (s_done) break;
        for (int step = 0; step < n - 1; step++) {
            // rotation of each disjoint pair of this round
            for (int k = t; k < n / 2; k += nt) {
                int p = rr_pos(k, step, n), q = rr_pos(n - 1 - k, step, n);
                if (p > q) {
                    const int x = p;
                    p = q;
                    q = x;
                }
                rp[k] = p;
                rq[k] = q;
                const double apq = A(p, q);
                double c = 1.0, s = 0.0;
                if (apq != 0.0) {
                    const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                    const double tt = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(tt * tt + 1.0);
                    s = tt * c;
                }
                rc[k] = c;
                rs[k] = s;
            }
            __syncthreads();
            // A <- A J and V <- V J (columns p, q of every row)
            for (int idx = t; idx < (n / 2) * n; idx += nt) {
                const int k = idx / n, r = idx % n;
                const int p = rp[k], q = rq[k];
                const double c = rc[k], s = rs[k];
                if (s == 0.0) continue;
                const double ap = A(r, p), aq = A(r, q);
                A(r, p) = c * ap - s * aq;
                A(r, q) = s * ap + c * aq;
                const double vp = V(r, p), vq = V(r, q);
                V(r, p) = c * vp - s * vq;
                V(r, q) = s * vp + c * vq;
            }
            __syncthreads();
            // A <- J^T A (rows p, q of every column)
            for (int idx = t; idx < (n / 2) * n; idx += nt) {
                const int k = idx / n, col = idx % n;
                const int p = rp[k], q = rq[k];
                const double c = rc[k], s = rs[k];
                if (s == 0.0) continue;
                const double ap = A(p, col), aq = A(q, col);
                A(p, col) = c * ap - s * aq;
                A(q, col) = s * ap + c * aq;
            }
            __syncthreads();
        }
    }
    // outputs: eigenvalues (times blen_mult), U = D^-1/2 V, U^-1 = V^T D^1/2
    double *lam = job.out, *U = lam + S, *Ui = U + S * S;
    for (int i = t; i < S; i += nt) lam[i] = A(i, i) * job.blen_mult;
    for (int idx = t; idx < S * S; idx += nt) {
        const int i = idx / S, k = idx % S;
        U[i * S + k] = V(i, k) / sq[i];
        Ui[k * S + i] = V(i, k) * sq[i];
    }
    if (t == 0 && job.sweeps) *job.sweeps = sweep;
#undef A
#undef V
}

}  // namespace gb
