// gb_dna.cuh -- 4-state (nucleotide) kernels of the garli_b200 engine.
//
// CLA layout in HBM is GARLI's: [pattern][rate][state] (tree.cpp:7669), one
// scaler int per pattern (condlike.h underflow_mult).  The plain form stores
// FP64 and evaluates every per-site expression in the reference's order with
// no fused multiply-add, so its CLAs are bit-identical to GARLI's CPU path
// given identical P matrices; the precision form stores FP32 and keeps each
// site's largest entry in [1,2) with an exact power-of-two rescale.
#pragma once
#include "gb_common.cuh"

namespace gb {

// 256-bit vector load/store of one (pattern, rate) 4-state slice (sm_100 ld/st.v4.f64)
__device__ __forceinline__ void ld4d(const double *p, double v[4]) {
    asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
                 : "l"(p));
}
__device__ __forceinline__ void st4d(double *p, const double v[4]) {
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
                 : "memory");
}
template <typename ST>
__device__ __forceinline__ void cla_load(const ST *p, double v[4]);
template <>
__device__ __forceinline__ void cla_load<double>(const double *p, double v[4]) { ld4d(p, v); }
// Stochastic rounding of a non-negative double to float: the lower or upper
// float neighbour with probability given by the position between them, the
// uniform variate being a hash of the value's address.  Unbiased and, unlike
// round-to-nearest, uncorrelated between patterns: the CLAs of small subtrees
// take few distinct values, and a deterministic rounding error of such a value
// would be repeated in every pattern that shares it and add up coherently in
// the lnL sum.  Deterministic (same address, same value -> same float).
// The gap hi - lo is one float ulp, a power of two, so the position
// (x - lo) / gap is formed exactly as a product with its reciprocal 2^(150-E)
// (E the float exponent field of lo; 2^149 below the normal range).  For x in
// [2^-126, 2^127) the same decision is taken on the bit fields: lo is x's
// sign, exponent and top 23 mantissa bits, and (x - lo) / gap is x's low 29
// mantissa bits over 2^29, so u < (x - lo) / gap iff (h >> 8) * 32 < those bits.
__device__ __forceinline__ unsigned int sr_hash(unsigned int key) {
    unsigned int h = key * 0x9E3779B1u;
    h ^= h >> 15;
    h *= 0x85EBCA77u;
    h ^= h >> 13;
    h *= 0xC2B2AE3Du;
    h ^= h >> 16;
    return h;
}
__device__ __forceinline__ float round_stochastic(double x, unsigned int key) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    const unsigned int eb = (unsigned int)(b >> 52);  // sign and exponent field
    if (eb >= 1023u - 126u && eb <= 1023u + 126u) {
        const unsigned int lo = ((eb - 896u) << 23) | (unsigned int)((b >> 29) & 0x7fffffu);
        return __uint_as_float(((sr_hash(key) >> 8) << 5) < (unsigned int)(b & 0x1fffffffu) ? lo + 1u : lo);
    }
    const float lo = __double2float_rz(x);
    const float hi = __int_as_float(__float_as_int(lo) + 1);
    if ((__float_as_uint(lo) >> 31) || !isfinite(hi)) return lo;
    const int E = (int)((__float_as_uint(lo) >> 23) & 0xffu);
    const double inv_gap = __longlong_as_double((long long)(1023 + (E ? 150 - E : 149)) << 52);
    const double frac = (x - (double)lo) * inv_gap;
    const double u = (double)(sr_hash(key) >> 8) * (1.0 / 16777216.0);
    return u < frac ? hi : lo;
}

// a slice of the edge kernels: FP64, or FP32 with its extension word e
template <typename ST>
__device__ __forceinline__ void cla_load_x(const ST *p, const unsigned int *e, double v[4]);
template <>
__device__ __forceinline__ void cla_load_x<double>(const double *p, const unsigned int *, double v[4]) { ld4d(p, v); }
template <>
__device__ __forceinline__ void cla_load_x<float>(const float *p, const unsigned int *e, double v[4]) {
    ext_decode4(__ldg(reinterpret_cast<const float4 *>(p)), __ldg(e), v);
}

template <typename ST>
__device__ __forceinline__ void cla_store(ST *p, const double v[4]);
template <>
__device__ __forceinline__ void cla_store<double>(double *p, const double v[4]) { st4d(p, v); }

// (a*b + c*d) + (e*f + g*h): the unrolled 4-rate kernels (tree.cpp:7705-7779, :8319-8376)
__device__ __forceinline__ double dot4_pair(const double *p, const double c[4]) {
    return add(add(mul(p[0], c[0]), mul(p[1], c[1])), add(mul(p[2], c[2]), mul(p[3], c[3])));
}
// ((a*b + c*d) + e*f) + g*h: the general-R kernels and the ambiguous-tip cases
__device__ __forceinline__ double dot4_seq(const double *p, const double c[4]) {
    return add(add(add(mul(p[0], c[0]), mul(p[1], c[1])), mul(p[2], c[2])), mul(p[3], c[3]));
}

// Tip classes of MakeAmbigStrings (sequencedata.cpp:278-363): a single state,
// total ambiguity (code -4) or a partial ambiguity listing its states in
// ascending order.
__device__ __forceinline__ int tip_class(int c) {
    c &= 15;
    if (c == 15 || c == 0) return 1;
    return (c & (c - 1)) ? 2 : 0;
}
// Value a terminal contributes for "from" state i: P[i][s] for one state,
// 0 + sum of P[i][s] over the listed states (tree.cpp:8004-8016), 1.0 when fully ambiguous.
__device__ __forceinline__ void tip_vec(const double *P, int c, double tv[4]) {
    c &= 15;
    if (c == 15 || c == 0) {
        tv[0] = tv[1] = tv[2] = tv[3] = 1.0;
        return;
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < 4; b++)
            if (c & (1 << b)) s = add(s, P[i * 4 + b]);
        tv[i] = s;
    }
}

// ---------------------------------------------------------------------------
// CLA update: one block = PPB patterns x G lanes (one lane per rate category),
// grid = (pattern tiles, ops of this dependency level).
//   Tree::CalcFullCLAInternalInternal   tree.cpp:7668
//   Tree::CalcFullCLAInternalTerminal   tree.cpp:8291
//   Tree::CalcFullCLATerminalTerminal   tree.cpp:7912
//   Tree::RescaleRateHet                tree.cpp:3370 (plain form, rank-gated)
// ---------------------------------------------------------------------------
template <typename ST, int R, bool GARLI_SCALE>
__device__ __forceinline__ void cla4_body(const View &v, const DevOp &op, const double *PL, const double *PR, int tile) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    const int r = threadIdx.x % G;
    const int p = tile * PPB + threadIdx.x / G;
    const bool act = (p < v.npat) && (r < R);
    double d[4] = {0.0, 0.0, 0.0, 0.0};
    int m = 0;
    if (act) {
        if (op.kind == kIntInt) {
            double a[4], b[4];
            cla_load<ST>(cla_ptr<ST>(v, op.c1, p, R * 4) + r * 4, a);
            cla_load<ST>(cla_ptr<ST>(v, op.c2, p, R * 4) + r * 4, b);
#pragma unroll
            for (int i = 0; i < 4; i++) {
                double L = (R == 4) ? dot4_pair(PL + 4 * i, a) : dot4_seq(PL + 4 * i, a);
                double Rr = (R == 4) ? dot4_pair(PR + 4 * i, b) : dot4_seq(PR + 4 * i, b);
                d[i] = mul(L, Rr);
            }
            if (r == 0) m = v.scalers[(long long)op.c1 * v.npat_pad + p] + v.scalers[(long long)op.c2 * v.npat_pad + p];
        } else if (op.kind == kIntTip) {
            double a[4];
            cla_load<ST>(cla_ptr<ST>(v, op.c1, p, R * 4) + r * 4, a);
            const int code = v.tips[(long long)op.c2 * v.npat_pad + p];
            const int cls = tip_class(code);
            if (cls == 0) {
                const int s = __ffs(code & 15) - 1;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    double L = (R == 4) ? dot4_pair(PL + 4 * i, a) : dot4_seq(PL + 4 * i, a);
                    // register-resident P: select column s without dynamic indexing
                    const double pr = s == 0 ? PR[4 * i] : s == 1 ? PR[4 * i + 1] : s == 2 ? PR[4 * i + 2] : PR[4 * i + 3];
                    d[i] = mul(L, pr);
                }
            } else if (cls == 1) {
#pragma unroll
                for (int i = 0; i < 4; i++) d[i] = dot4_seq(PL + 4 * i, a);
            } else {
                double tv[4];
                tip_vec(PR, code, tv);
#pragma unroll
                for (int i = 0; i < 4; i++) d[i] = mul(tv[i], dot4_seq(PL + 4 * i, a));
            }
            if (r == 0) m = v.scalers[(long long)op.c1 * v.npat_pad + p];
        } else {
            double tl[4], tr[4];
            tip_vec(PL, v.tips[(long long)op.c1 * v.npat_pad + p], tl);
            tip_vec(PR, v.tips[(long long)op.c2 * v.npat_pad + p], tr);
#pragma unroll
            for (int i = 0; i < 4; i++) d[i] = mul(tl[i], tr[i]);
        }
    }
    if (GARLI_SCALE) {
        if (op.rescale) {
            double mx = act ? fmax(fmax(d[0], d[2]), fmax(d[1], d[3])) : 0.0;
#pragma unroll
            for (int o = 1; o < G; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (act && mx < c_rescale_below) {
                if (mx < c_reduce_below && (v.rescale_every > 2 || mx < c_bail_below)) {
                    if (r == 0) atomicOr(v.status, kStatusRescaleRetry);
                }
                int idx = 0;
                while ((idx + 1) < kRescaleTableLen && c_thresh[idx + 1] > mx) idx++;
                const double mu = c_mult[idx];
#pragma unroll
                for (int i = 0; i < 4; i++) d[i] = mul(d[i], mu);
                m += c_incr[idx];
            }
        }
    } else {
        double mx = act ? fmax(fmax(d[0], d[2]), fmax(d[1], d[3])) : 0.0;
#pragma unroll
        for (int o = 1; o < G; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (act && mx > 0.0) {
            const int e = ilogb(mx);
            const double sc = ldexp(1.0, -e);
#pragma unroll
            for (int i = 0; i < 4; i++) d[i] *= sc;
            m -= e;
        }
    }
    if (act) {
        cla_store<ST>(cla_ptr<ST>(v, op.dest, p, R * 4) + r * 4, d);
        if (r == 0) v.scalers[(long long)op.dest * v.npat_pad + p] = m;
    }
}

// P(t) of this lane's rate category for both children stay in registers; the
// block walks its share of pattern tiles (grid-stride), so the per-block setup
// is amortised over many tiles.
template <int R, bool GARLI_SCALE>
__global__ void __launch_bounds__(kThreads) k_cla4(View v, LevelOps ops) {
    constexpr int G = Lanes<R>::G;
    constexpr int PPB = kThreads / G;
    const DevOp op = ops.op[blockIdx.y];
    const int r = threadIdx.x % G;
    const int rr = r < R ? r : 0;
    double PL[16], PR[16];
    {
        const double *m1 = v.mats + (long long)op.p1 * v.mat_stride + 16 * rr;
        const double *m2 = v.mats + (long long)op.p2 * v.mat_stride + 16 * rr;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            PL[i] = __ldg(m1 + i);
            PR[i] = __ldg(m2 + i);
        }
    }
    const int ntiles = (v.npat + PPB - 1) / PPB;
    // the plain form keeps every pattern in FP64 (the precision form's CLA
    // updates are k_cla4m / k_level4m)
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) cla4_body<double, R, GARLI_SCALE>(v, op, PL, PR, tile);
}

// Block-level sum of three doubles; thread 0 writes the block's partial sums.
__device__ __forceinline__ void block_sum3(double a, double b, double c, double *out) {
    __shared__ double red[3][kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) {
        red[0][w] = a;
        red[1][w] = b;
        red[2][w] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int i = 0; i < (int)(blockDim.x / 32); i++) {
            s0 += red[0][i];
            s1 += red[1][i];
            s2 += red[2][i];
        }
        out[0] = s0;
        out[1] = s1;
        out[2] = s2;
    }
}

// ---------------------------------------------------------------------------
// Edge evaluation: per-pattern site likelihood (and dL/dt, d2L/dt2) across a
// branch, count-weighted lnL (and d1, d2) partial sums per block.
//   Tree::GetScorePartialInternalRateHet  tree.cpp:6172
//   Tree::GetScorePartialTerminalRateHet  tree.cpp:6040
//   Tree::GetDerivsPartialInternal        optimization.cpp:3063
//   Tree::GetDerivsPartialTerminal        optimization.cpp:2412
// One thread per pattern; the rate loop runs in the reference's order.
// ---------------------------------------------------------------------------
template <int R, bool DERIV>
struct EdgeSmem {
    __align__(16) double M[3][R * 16];
    double F[4], RP[R];
};

template <typename ST, int R, bool GARLI_SCALE, bool DERIV>
__device__ __forceinline__ void edge4_site(const View &v, const EdgeSmem<R, DERIV> &sm, int pbuf, int cbuf,
                                           int child_tip, int write_sites, int p, double &accL, double &acc1,
                                           double &acc2) {
    const double *f = sm.F;
    double L[4] = {0, 0, 0, 0}, D1[4] = {0, 0, 0, 0}, D2[4] = {0, 0, 0, 0};
    const int m1 = v.scalers[(long long)pbuf * v.npat_pad + p];
    const int m2 = child_tip ? 0 : v.scalers[(long long)cbuf * v.npat_pad + p];
    const ST *PC = cla_ptr<ST>(v, pbuf, p, R * 4);
    // the FP32 segment's extension words (precision form)
    const unsigned int *PE = nullptr, *CE = nullptr;
    if constexpr (sizeof(ST) == 4) {
        PE = cla_ext(v, pbuf, p, R * 4);
        if (!child_tip) CE = cla_ext(v, cbuf, p, R * 4);
    }
    if (!child_tip) {
        const ST *CC = cla_ptr<ST>(v, cbuf, p, R * 4);
#pragma unroll
        for (int r = 0; r < R; r++) {
            double part[4], c[4];
            cla_load_x<ST>(PC + r * 4, PE + r, part);
            cla_load_x<ST>(CC + r * 4, CE + r, c);
            const double rp = sm.RP[r];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                L[i] = add(L[i], mul(mul(dot4_seq(&sm.M[0][16 * r + 4 * i], c), part[i]), rp));
                if (DERIV) {
                    D1[i] = add(D1[i], mul(mul(dot4_seq(&sm.M[1][16 * r + 4 * i], c), part[i]), rp));
                    D2[i] = add(D2[i], mul(mul(dot4_seq(&sm.M[2][16 * r + 4 * i], c), part[i]), rp));
                }
            }
        }
    } else {
        const int code = v.tips[(long long)cbuf * v.npat_pad + p] & 15;
        const int cls = tip_class(code);
        if (cls == 1) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                double part[4];
                cla_load_x<ST>(PC + r * 4, PE + r, part);
#pragma unroll
                for (int i = 0; i < 4; i++) L[i] = add(L[i], mul(part[i], sm.RP[r]));
            }
        } else {
            // single state: one pass; partial ambiguity: states outer, rates inner
            for (int s = 0; s < 4; s++) {
                if (!(code & (1 << s))) continue;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    double part[4];
                    cla_load_x<ST>(PC + r * 4, PE + r, part);
                    const double rp = sm.RP[r];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        L[i] = add(L[i], mul(mul(sm.M[0][16 * r + 4 * i + s], part[i]), rp));
                        if (DERIV) {
                            D1[i] = add(D1[i], mul(mul(sm.M[1][16 * r + 4 * i + s], part[i]), rp));
                            D2[i] = add(D2[i], mul(mul(sm.M[2][16 * r + 4 * i + s], part[i]), rp));
                        }
                    }
                }
            }
        }
    }
    double siteL = add(add(add(mul(L[0], f[0]), mul(L[1], f[1])), mul(L[2], f[2])), mul(L[3], f[3]));
    const int cb = v.const_states[p];
    if (v.has_pinv && cb >= 0) {
        double btot = 0.0;
        if (cb & 1) btot = add(btot, f[0]);
        if (cb & 2) btot = add(btot, f[1]);
        if (cb & 4) btot = add(btot, f[2]);
        if (cb & 8) btot = add(btot, f[3]);
        if (GARLI_SCALE) {
            if (DERIV) {
                // (prI*btot)*exp(child + partial) (optimization.cpp:2540, :3166)
                const double e = child_tip ? exp((double)m1) : exp(add((double)m2, (double)m1));
                siteL = add(siteL, mul(mul(v.pinv, btot), e));
            } else if (m1 + m2 == 0) {
                siteL = add(siteL, mul(v.pinv, btot));
            } else {
                // prI*btot*exp(partial + child) (tree.cpp:6128, :6236)
                siteL = add(siteL, mul(mul(v.pinv, btot), exp(add((double)m1, (double)m2))));
            }
        } else {
            siteL = add(siteL, ldexp(mul(v.pinv, btot), m1 + m2));
        }
    }
    double u;
    if (GARLI_SCALE) {
        const double lg = log(siteL);
        if (DERIV && !child_tip) u = sub(sub(lg, (double)m2), (double)m1);
        else u = sub(sub(lg, (double)m1), (double)m2);
    } else {
        u = sub(log(siteL), (double)(m1 + m2) * 0.69314718055994530941723212145818);
    }
    const double cnt = (double)v.counts[p];
    accL = add(accL, mul(cnt, u));
    if (DERIV) {
        const double sd1 = add(add(add(mul(D1[0], f[0]), mul(D1[1], f[1])), mul(D1[2], f[2])), mul(D1[3], f[3])) / siteL;
        const double sd2 =
            sub(add(add(add(mul(D2[0], f[0]), mul(D2[1], f[1])), mul(D2[2], f[2])), mul(D2[3], f[3])) / siteL,
                mul(sd1, sd1));
        acc1 = add(acc1, mul(cnt, sd1));
        acc2 = add(acc2, mul(cnt, sd2));
        if (write_sites) {
            v.site_d1[p] = sd1;
            v.site_d2[p] = sd2;
        }
    }
    if (write_sites) v.site_lnl[p] = u;
}

template <int R, bool DERIV>
__device__ __forceinline__ void edge4_load_smem(const View &v, int mat, EdgeSmem<R, DERIV> &sm) {
    const double *mp = v.mats + (long long)mat * v.mat_stride;
    for (int i = threadIdx.x; i < R * 16; i += blockDim.x) {
        sm.M[0][i] = mp[i];
        if (DERIV) {
            sm.M[1][i] = mp[R * 16 + i];
            sm.M[2][i] = mp[2 * R * 16 + i];
        }
    }
    if (threadIdx.x < 4) sm.F[threadIdx.x] = v.freqs[threadIdx.x];
    if (threadIdx.x < R) sm.RP[threadIdx.x] = v.rate_probs[threadIdx.x];
}

template <int R, bool GARLI_SCALE, bool DERIV>
__global__ void __launch_bounds__(kThreads) k_edge4(View v, int pbuf, int cbuf, int mat, int child_tip,
                                                    int write_sites) {
    __shared__ EdgeSmem<R, DERIV> sm;
    edge4_load_smem<R, DERIV>(v, mat, sm);
    __syncthreads();
    double accL = 0.0, acc1 = 0.0, acc2 = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < v.npat; p += gridDim.x * blockDim.x) {
        if (p < v.kpad)
            edge4_site<double, R, GARLI_SCALE, DERIV>(v, sm, pbuf, cbuf, child_tip, write_sites, p, accL, acc1, acc2);
        else
            edge4_site<float, R, GARLI_SCALE, DERIV>(v, sm, pbuf, cbuf, child_tip, write_sites, p, accL, acc1, acc2);
    }
    block_sum3(accL, acc1, acc2, v.block_sums + 3 * blockIdx.x);
}

}  // namespace gb
