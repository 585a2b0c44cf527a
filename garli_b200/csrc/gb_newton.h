// gb_newton.h -- one iteration of GARLI's Newton-Raphson branch-length optimiser
// as a state machine shared by the host tree driver and the device graph.
//
// Restates Tree::NewtonRaphsonOptimizeBranchLength (optimization.cpp:1359-1971,
// FP64 build, default exit rule, OPT_DEBUG off).  One call consumes the
// derivatives (d1, d2) and lnL evaluated at the current length and either
// finishes (the current length, or the entry length when GARLI restores it,
// is final) or proposes the next length.  Two places where GARLI rescores
// the tree with Score() use the lnL of the derivative evaluation at the same
// length instead (the same quantity, equal to rounding): the "score worsened
// at the minimum length" restore (:1538-1551) and the 100-pass guard
// (:1894-1936).  Arithmetic is spelled out without fused multiply-add so the
// host and the device produce identical decisions.
#pragma once
#include <cfloat>
#include <cmath>

#ifdef __CUDACC__
#define GB_HD __host__ __device__ __forceinline__
#else
#define GB_HD inline
#endif

namespace gb {

#ifdef __CUDA_ARCH__
GB_HD double nmul(double a, double b) { return __dmul_rn(a, b); }
GB_HD double nadd(double a, double b) { return __dadd_rn(a, b); }
GB_HD double nsub(double a, double b) { return __dsub_rn(a, b); }
#else
GB_HD double nmul(double a, double b) {
    volatile double r = a * b;
    return r;
}
GB_HD double nadd(double a, double b) {
    volatile double r = a + b;
    return r;
}
GB_HD double nsub(double a, double b) {
    volatile double r = a - b;
    return r;
}
#endif

struct NrState {
    double v, v_prev, v_onEntry, knownMin, knownMax, initialL, totalEstImprove;
    int iter, negProposalNum, done, final_check;
};

GB_HD void nr_init(NrState &s, double dlen, double min_brlen, double max_brlen) {
    s.v = s.v_prev = s.v_onEntry = dlen;
    s.knownMin = min_brlen;
    s.knownMax = max_brlen;
    s.initialL = 0.0;
    s.totalEstImprove = 0.0;
    s.iter = 0;
    s.negProposalNum = 0;
    s.done = 0;
    s.final_check = 0;
}

GB_HD bool nr_feq(double a, double b, double eps) { return fabs(a - b) < eps; }

// delta*d1 + (delta*delta*d2*0.5): scoreDeltaToMin/Max and the totalEstImprove
// increments (optimization.cpp:1712, :1747, :1781, :1800)
GB_HD double nr_quad(double delta, double d1, double d2) {
    return nadd(nmul(delta, d1), nmul(nmul(nmul(delta, delta), d2), 0.5));
}
// d1*delta + (d2*delta*delta*0.5): estImp of the wrong-curvature branch (:1569, :1599)
GB_HD double nr_quad_est(double delta, double d1, double d2) {
    return nadd(nmul(d1, delta), nmul(nmul(nmul(d2, delta), delta), 0.5));
}

// Returns 1 when the optimisation of this branch is finished (final length in
// s.v), 0 when s.v holds the next length to evaluate.
GB_HD int nr_step(NrState &s, double d1, double d2, double lnL, double precision1, double min_brlen,
                  double max_brlen) {
    const double dlen = s.v;
    if (s.final_check) {
        // 100-pass guard (optimization.cpp:1894-1936): keep the length if lnL improved
        s.done = 1;
        if (!(lnL > s.initialL)) {
            s.v = s.v_onEntry;
            s.totalEstImprove = 0.0;
        }
        return 1;
    }
    if (s.iter == 0) s.initialL = lnL;
    const double estDeltaNR = -d1 / d2;
    const double estScoreDelta = nadd(nmul(d1, estDeltaNR), nmul(nmul(nmul(d2, estDeltaNR), estDeltaNR), 0.5));
    if (d1 <= 0.0 && dlen < s.knownMax) s.knownMax = dlen;
    else if (d1 > 0.0 && dlen > s.knownMin) s.knownMin = dlen;
    double v = s.v;
    if (d2 >= 0.0) {
        double proposed;
        if (d1 <= 0.0) {
            if (nr_feq(dlen, min_brlen, 1.0e-8)) {
                if (lnL < nsub(s.initialL, pow(10.0, -6.0 + ceil(log10(-lnL))))) {
                    s.v = s.v_onEntry;
                    s.totalEstImprove = 0.0;
                }
                s.done = 1;
                return 1;
            }
            if (s.knownMin == min_brlen) {
                if (dlen <= 1.0e-4) proposed = min_brlen;
                else if (dlen <= 0.005) proposed = 1.0e-4;
                else if (dlen <= 0.05) proposed = nmul(dlen, 0.1);
                else proposed = nmul(dlen, 0.25);
            } else
                proposed = nmul(nadd(s.knownMin, dlen), 0.5);
            if (s.iter > 0 || proposed == min_brlen) {
                const double estImp = nr_quad_est(nsub(proposed, dlen), d1, d2);
                if (estImp < precision1 && lnL >= nsub(s.initialL, 1.0e-4)) {
                    s.done = 1;
                    return 1;
                }
            }
        } else {
            if (s.knownMax == max_brlen) {
                if (dlen < 0.1) proposed = nmul(dlen, 10.0);
                else proposed = fmin(nmul(dlen, 2.0), max_brlen);
            } else
                proposed = nmul(nadd(s.knownMax, dlen), 0.5);
            if (s.iter > 0) {
                const double estImp = nr_quad_est(nsub(proposed, dlen), d1, d2);
                if (estImp < precision1 && lnL >= nsub(s.initialL, 1.0e-4)) {
                    s.done = 1;
                    return 1;
                }
            }
        }
        v = proposed;
        s.totalEstImprove = nadd(s.totalEstImprove, precision1);
    } else {
        if (d1 < 0.0 && nr_feq(dlen, min_brlen, 1.0e-8)) {
            s.done = 1;
            return 1;
        }
        if (d1 > 0.0 && nr_feq(dlen, max_brlen, 1.0e-8)) {
            s.done = 1;
            return 1;
        }
        const double tol = nmul((double)(s.iter < 10 ? 1 : s.iter), fmax(1.0e-7, DBL_EPSILON * 10.0));
        if (estScoreDelta < precision1 && (s.iter == 0 || nadd(lnL, tol) >= s.initialL)) {
            s.done = 1;
            return 1;
        }
        bool noNR = false;
        if (s.iter > 10) {
            if (d1 > 0.0) {
                if (nr_feq(s.knownMax, max_brlen, 1e-8)) {
                    if ((s.iter > 20) && (dlen > (max_brlen / 2.0))) v = max_brlen;
                    else if (v < 0.2) v = fmin(nmul(nadd(v, max_brlen), 0.5), nmul(v, 5.0));
                    else v = fmin(nmul(nadd(v, max_brlen), 0.5), nmul(v, 2.0));
                    noNR = true;
                } else if (((s.iter - 20) > 0) && ((s.iter - 20) % 10 == 0)) {
                    v = fmin(nmul(nadd(v, s.knownMax), 0.5), nmul(v, 100.0));
                }
            } else if (nr_feq(s.knownMin, min_brlen, 1e-8)) {
                v = (s.iter > 20) ? min_brlen : nmul(nadd(v, min_brlen), 0.5);
                noNR = true;
            }
        }
        if (!noNR) v = nadd(v, estDeltaNR);
        if (v <= s.knownMin) {
            s.negProposalNum++;
            if (s.knownMin == min_brlen) {
                const double sdm = nr_quad(nsub(min_brlen, dlen), d1, d2);
                if (sdm < precision1) {
                    s.done = 1;
                    return 1;
                }
                if (s.negProposalNum == 1 && dlen > 1e-4 && s.v_prev != 1e-4) {
                    if (dlen < .005) v = 1e-4;
                    else if (dlen < 0.05) v = nmul(dlen, 0.1);
                    else v = nmul(dlen, 0.25);
                    s.totalEstImprove = nadd(s.totalEstImprove, nr_quad(nsub(v, dlen), d1, d2));
                } else {
                    v = min_brlen;
                    s.totalEstImprove = nadd(s.totalEstImprove, sdm);
                }
            } else {
                const double proposed = nmul(nadd(s.knownMin, dlen), 0.5);
                const double sdm = nr_quad(nsub(proposed, dlen), d1, d2);
                if (sdm < precision1) {
                    s.done = 1;
                    return 1;
                }
                v = proposed;
                s.totalEstImprove = nadd(s.totalEstImprove, sdm);
            }
        } else if (v >= s.knownMax) {
            if (s.knownMax == max_brlen) {
                const double sdm = nr_quad(nsub(max_brlen, dlen), d1, d2);
                if (sdm < precision1) {
                    s.done = 1;
                    return 1;
                }
                v = max_brlen;
                s.totalEstImprove = nadd(s.totalEstImprove, sdm);
            } else {
                const double proposed = nmul(nadd(s.knownMax, dlen), 0.5);
                const double sdm = nr_quad(nsub(proposed, dlen), d1, d2);
                if (sdm < precision1) {
                    s.done = 1;
                    return 1;
                }
                v = proposed;
                s.totalEstImprove = nadd(s.totalEstImprove, sdm);
            }
        } else
            s.totalEstImprove = nadd(s.totalEstImprove, estScoreDelta);
    }
    // SetBranchLength(nd, v) is the caller's; then the 100-pass guard
    s.v = v;
    s.v_prev = v;
    s.iter++;
    if (s.iter > 100) s.final_check = 1;
    return 0;
}

}  // namespace gb
