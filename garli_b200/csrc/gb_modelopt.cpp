// gb_modelopt.cpp -- GARLI's model-parameter optimisation on top of the tree layer.
//
// Restates, for one tree and its model:
//   * the parameter setters the optimiser calls: Model::SetAlpha (model.h:1742,
//     DiscreteGamma model.cpp:2170-2201), SetPinv (model.h:1733),
//     SetEquilibriumFreq with NormalizeSumConstrainedValues (model.h:1501-1516,
//     :1681-1731), SetRelativeNucRate (model.h:1518-1531), SetOmega (model.h:1797);
//   * Tree::OptimizeBoundedParameter (optimization.cpp:332-776) as compiled by
//     default (NEW_BUMPING and ADAPTIVE_BOUNDED_OPT on, defs.h:63-67; double
//     precision: STEP_TOL 1e-8, optimization.cpp:33-39) with
//     SetAndEvaluateParameter (:244-268) and CheckScoreAndRestore (:271-301);
//   * its callers with their bounds: alpha and pinv (population.cpp:2702, :2727),
//     Tree::OptimizeEquilibriumFreqs (tree.cpp:7288-7305),
//     Tree::OptimizeRelativeNucRates (tree.cpp:7307-7355, nucleotide and codon
//     rate matrices), single-class omega (tree.cpp:7186-7191);
//   * Population::BetterFinalOptimization (population.cpp:2566-2790).
//
// Every SetAndEvaluateParameter is a full rescore under a new model.  The
// optimiser keeps GARLI's sequence of evaluations and decisions; what it adds
// is that evaluation points whose values are known before their scores are
// needed are scored in one gbt_score_models call (one levelled CLA pass over
// all of them, their eigen systems in one gb_set_eigen_from_rate_matrices
// launch):
//   pass 0      the bumped start value, then the first higher / lower points
//               and, speculatively, the higher / lower points of the next
//               adaptive increment widenings (ADAPTIVE_BOUNDED_OPT);
//   pass p > 0  the proposed value of pass p-1 together with the higher and
//               lower points of pass p, whose increment is fixed once the
//               brackets are updated (no widening after pass 0).
// A speculative score that GARLI would not have computed is never used, and
// each point's model is built along the chain of setter calls GARLI makes to
// reach it (SetEquilibriumFreq renormalises the model it is given, so the
// chain matters in the last bits): the batching changes no result.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/garli_b200.h"

namespace {

const double kStepTol = 1.0e-8;      // STEP_TOL, double precision (optimization.cpp:33-39)
const double kFpEps = 2.220446049250313e-16;  // DBL_EPSILON (GARLI_FP_EPS, defs.h:109)

struct Opt {
    int tree = -1, inst = -1;
    gb_model_params m{};        // the tree's model (GARLI's Model after the last setter call)
    std::vector<double> exch;   // fixed amino-acid exchangeabilities
    double lnL = -1.0;          // Tree::lnL (-1: unknown)
    int kmax = 1;               // models one gbt_score_models call can take
    int depth = 3;              // 0: no batching; 1: known points; >= 2: + speculative widenings (depth - 1 of them)
    long long evals = 0, scored = 0, calls = 0;
    // evaluations of the last OptimizeBoundedParameter call, in GARLI's order
    double traceInitial = 0.0;
    std::vector<double> traceVal, traceScore;
};

std::mutex g_mu;
std::vector<Opt *> g_opts;

Opt *get(int h) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h < 0 || h >= (int)g_opts.size()) return nullptr;
    return g_opts[h];
}

bool fp_equals(double a, double b, double eps) { return std::fabs(a - b) < eps; }

// ---- setters (model.h) ----

// Model::NormalizeSumConstrainedValues (model.h:1681-1731)
void normalize_sum_constrained(double *v, int n, double target, double minVal, int keep) {
    bool someMin = false;
    double minSum = 0.0, sum = 0.0;
    for (int i = 0; i < n; i++)
        if (i != keep) {
            sum += v[i];
            if (v[i] < minVal) someMin = true;
        }
    if (someMin || !fp_equals(sum, target, minVal * 0.01)) {
        do {
            const double unfixed = target - (keep < 0 ? 0.0 : v[keep]) - minSum;
            const double rescale = unfixed / sum;
            someMin = false;
            sum = 0.0;
            for (int i = 0; i < n; i++) {
                if (i == keep || !(v[i] > 0.0)) continue;
                v[i] *= rescale;
                if (v[i] < minVal) {
                    v[i] = -1.0;
                    minSum += minVal;
                    someMin = true;
                } else {
                    sum += v[i];
                }
            }
        } while (someMin);
    }
    for (int i = 0; i < n; i++)
        if (v[i] < 0.0) v[i] = minVal;
}

// the rate classes sharing relative rate `which` (nst 2: transitions AG, CT / transversions)
void set_rel_rate(gb_model_params &m, int which, double val) {
    if (m.nst == 2) {
        const bool ts = which == 1 || which == 4;
        for (int i = 0; i < 6; i++)
            if ((i == 1 || i == 4) == ts) m.rel[i] = val;
    } else {
        m.rel[which] = val;
    }
    // Model::SetRelativeNucRate: keep the reference rate (GT) at 1
    if (!fp_equals(m.rel[5], 1.0, 1.0e-12)) {
        const double scaler = 1.0 / m.rel[5];
        for (int i = 0; i < 5; i++) m.rel[i] *= scaler;
        m.rel[5] *= scaler;
    }
}

void apply(gb_model_params &m, int param, int which, double val) {
    switch (param) {
    case GB_PARAM_ALPHA: m.alpha = val; break;
    case GB_PARAM_PINV: m.pinv = val; break;
    case GB_PARAM_STATE_FREQ:
        m.pi[which] = val;
        normalize_sum_constrained(m.pi, m.stateCount, 1.0, 1e-4, which);
        break;
    case GB_PARAM_REL_RATE: set_rel_rate(m, which, val); break;
    case GB_PARAM_OMEGA: m.omega = val; break;
    }
}

double get_param(const gb_model_params &m, int param, int which) {
    switch (param) {
    case GB_PARAM_ALPHA: return m.alpha;
    case GB_PARAM_PINV: return m.pinv;
    case GB_PARAM_STATE_FREQ: return m.pi[which];
    case GB_PARAM_REL_RATE: return m.rel[which];
    default: return m.omega;
    }
}

bool valid_param(const gb_model_params &m, int param, int which) {
    switch (param) {
    case GB_PARAM_ALPHA: return m.categoryCount > 1;
    case GB_PARAM_PINV: return m.hasPinv != 0;
    case GB_PARAM_STATE_FREQ: return which >= 0 && which < m.stateCount;
    case GB_PARAM_REL_RATE: return m.kind != GB_MODEL_AMINO_ACID && m.nst > 1 && which >= 0 && which < 5;
    case GB_PARAM_OMEGA: return m.kind == GB_MODEL_CODON;
    }
    return false;
}

// ---- a model on the engine ----

struct Built {
    std::vector<double> Q, rates, weights;
    double blenMult = 1.0;
};

int build(const Opt &o, const gb_model_params &m, Built &b) {
    const int S = m.stateCount, R = m.categoryCount;
    b.Q.assign((size_t)S * S, 0.0);
    int rc;
    if (m.kind == GB_MODEL_NUCLEOTIDE) rc = gbm_gtr_qmat(m.rel, m.pi, b.Q.data(), &b.blenMult);
    else if (m.kind == GB_MODEL_AMINO_ACID) rc = gbm_aa_qmat(o.exch.data(), m.pi, b.Q.data(), &b.blenMult);
    else rc = gbm_codon_qmat6(m.rel, m.omega, m.pi, b.Q.data(), &b.blenMult);
    if (rc) return rc;
    b.rates.assign(R, 1.0);
    if (R > 1 && (rc = gbm_discrete_gamma(m.alpha, R, b.rates.data()))) return rc;
    const double pinv = m.hasPinv ? m.pinv : 0.0;
    b.weights.assign(R, (1.0 - pinv) / R);  // DiscreteGamma / SetPinv rateProbs
    return GB_SUCCESS;
}

// models ms into eigen / model slots first .. first+n-1
int upload(Opt &o, const std::vector<gb_model_params> &ms, int first) {
    const int n = (int)ms.size();
    if (n == 0) return GB_SUCCESS;
    const int S = ms[0].stateCount;
    std::vector<Built> b(n);
    std::vector<double> Q, pi, bm;
    std::vector<int> slots(n);
    for (int k = 0; k < n; k++) {
        int rc = build(o, ms[k], b[k]);
        if (rc) return rc;
        Q.insert(Q.end(), b[k].Q.begin(), b[k].Q.end());
        pi.insert(pi.end(), ms[k].pi, ms[k].pi + S);
        bm.push_back(b[k].blenMult);
        slots[k] = first + k;
    }
    int rc = gb_set_eigen_from_rate_matrices(o.inst, n, slots.data(), Q.data(), pi.data(), bm.data(), nullptr);
    if (rc) return rc;
    for (int k = 0; k < n; k++) {
        const double pinv = ms[k].hasPinv ? ms[k].pinv : 0.0;
        rc = gb_set_model_slot(o.inst, slots[k], ms[k].pi, b[k].rates.data(), b[k].weights.data(), pinv,
                               ms[k].hasPinv);
        if (rc) return rc;
    }
    return GB_SUCCESS;
}

// the model of the tree itself (slot 0); its CLAs become dirty
int install(Opt &o, const gb_model_params &m) {
    int rc = upload(o, std::vector<gb_model_params>{m}, 0);
    if (rc) return rc;
    o.m = m;
    return gbt_make_all_dirty(o.tree);
}

// full rescores of the tree under each model (slots 1..), kmax at a time
int score_batch(Opt &o, const std::vector<gb_model_params> &ms, std::vector<double> &lnl) {
    lnl.assign(ms.size(), 0.0);
    for (size_t s = 0; s < ms.size(); s += o.kmax) {
        const int n = (int)std::min<size_t>(o.kmax, ms.size() - s);
        std::vector<gb_model_params> part(ms.begin() + s, ms.begin() + s + n);
        int rc = upload(o, part, 1);
        if (rc) return rc;
        std::vector<int> slots(n);
        for (int k = 0; k < n; k++) slots[k] = 1 + k;
        rc = gbt_score_models(o.tree, n, slots.data(), lnl.data() + s);
        if (rc) return rc;
        o.scored += n;
        o.calls++;
    }
    return GB_SUCCESS;
}

int score_current(Opt &o) {
    double out[3];
    int rc = gbt_score(o.tree, 0, out);
    if (rc) return rc;
    o.lnL = out[0];
    return GB_SUCCESS;
}

// ---- Tree::OptimizeBoundedParameter (optimization.cpp:332-776) ----

struct Bounded {
    Opt &o;
    const int param, which;
    // scores computed ahead of their evaluation, by value, with the model each was computed for
    struct Ahead {
        gb_model_params m;
        double lnl;
    };
    std::map<double, Ahead> ahead;
    double bestKnownScore = 0.0, bestKnownVal = 0.0;

    Bounded(Opt &opt, int p, int w) : o(opt), param(p), which(w) {}

    gb_model_params with(double val) const {
        gb_model_params m = o.m;
        apply(m, param, which, val);
        return m;
    }

    // An evaluation point scored ahead: its value and the point evaluated just
    // before it on the path the optimiser will take if it reaches it (an index
    // into the same list; -1: the current model), so that its model is the one
    // GARLI's chain of setter calls gives.
    struct Pt {
        double v;
        int after;
    };
    // score the points in one batch; earlier speculation is dropped
    int prefetch(const std::vector<Pt> &pts) {
        if (o.depth == 0) return GB_SUCCESS;
        ahead.clear();
        std::vector<gb_model_params> ms(pts.size());
        for (size_t k = 0; k < pts.size(); k++) {
            ms[k] = pts[k].after < 0 ? o.m : ms[pts[k].after];
            apply(ms[k], param, which, pts[k].v);
        }
        std::vector<double> lnl;
        int rc = score_batch(o, ms, lnl);
        if (rc) return rc;
        for (size_t k = 0; k < pts.size(); k++) ahead.emplace(pts[k].v, Ahead{ms[k], lnl[k]});
        return GB_SUCCESS;
    }

    // SetAndEvaluateParameter (optimization.cpp:244-268): a point scored ahead
    // is used once, else the model is scored now
    int evaluate(double val, double *score) {
        auto it = ahead.find(val);
        Ahead a;
        if (it != ahead.end()) {
            a = it->second;
            ahead.erase(it);
        } else {
            std::vector<gb_model_params> ms{with(val)};
            std::vector<double> lnl;
            int rc = score_batch(o, ms, lnl);
            if (rc) return rc;
            a = Ahead{ms[0], lnl[0]};
        }
        o.m = a.m;
        o.lnL = a.lnl;
        o.evals++;
        o.traceVal.push_back(val);
        o.traceScore.push_back(o.lnL);
        if (o.lnL > bestKnownScore) {
            bestKnownVal = val;
            bestKnownScore = o.lnL;
        }
        *score = o.lnL;
        return GB_SUCCESS;
    }

    // CheckScoreAndRestore (optimization.cpp:271-301): the parameter takes
    // bestVal if it scores above otherScore + tolerance, else otherVal
    int check_score_and_restore(double otherScore, double otherVal, double bestScore, double bestVal,
                                double tolerance) {
        double v = otherVal;
        if (otherScore + tolerance < bestScore) {
            v = bestVal;
            otherScore = bestScore;
        }
        gb_model_params m = o.m;
        apply(m, param, which, v);
        int rc = install(o, m);
        if (rc) return rc;
        o.lnL = otherScore;
        return GB_SUCCESS;
    }

    // the increments of pass 0: the first, then each adaptive widening up to the bracket limit
    static std::vector<double> pass0_increments(double baseIncr, double incrLimit, int levels) {
        std::vector<double> inc;
        if (baseIncr > incrLimit) {
            inc.push_back(incrLimit / 1.0001);
            return inc;
        }
        inc.push_back(baseIncr);
        double b = baseIncr;
        for (int j = 1; j < levels; j++) {
            b *= 5.0;
            if (b > incrLimit) {
                inc.push_back(incrLimit / 1.0001);
                break;
            }
            inc.push_back(b);
        }
        return inc;
    }

    int run(double optPrecision, double initialVal, double lowBound, double highBound, double targetScoreDigits,
            double *result) {
        int rc;
        if (fp_equals(o.lnL, -1.0, std::max(1.0e-8, kFpEps * 2.0)) && (rc = score_current(o))) return rc;
        double baseIncr = std::min(std::max(0.001 * optPrecision, 1.0e-6), initialVal * 0.01);
        double curVal = initialVal;
        const double initialScore = o.lnL;
        o.traceInitial = initialScore;
        o.traceVal.clear();
        o.traceScore.clear();
        double curScore = initialScore;
        bestKnownScore = initialScore;
        bestKnownVal = initialVal;
        *result = 0.0;

        // NEW_BUMPING
        const double requiredWindow = (baseIncr * 1.0001) * 2.0;
        const double actualWindow = highBound - lowBound;
        if (actualWindow < requiredWindow) return GB_SUCCESS;
        double boundBumped = -1.0;
        double bumpAmt = baseIncr * 25.0001;
        bool bump = false;
        if (lowBound + bumpAmt > initialVal) {
            if (lowBound + bumpAmt > highBound - bumpAmt) bumpAmt = actualWindow / 2.0;
            boundBumped = std::fabs(curVal - (lowBound + bumpAmt));
            curVal = lowBound + bumpAmt;
            bump = true;
        } else if (highBound - bumpAmt < initialVal) {
            if (highBound - bumpAmt < lowBound + bumpAmt) bumpAmt = actualWindow / 2.0;
            curVal = highBound - bumpAmt;
            boundBumped = initialVal - curVal;
            bump = true;
        }
        double upperBracket = highBound, lowerBracket = lowBound;
        {
            // pass 0's points are known now: the bumped value, the first pair and
            // (speculatively) the pairs of the adaptive widenings; GARLI's path
            // through them is bump, higher_0, .., higher_J, lower_J
            std::vector<Pt> pts;
            int prev = -1;
            if (bump) {
                pts.push_back({curVal, -1});
                prev = 0;
            }
            const double incrLimit = std::min(curVal - lowerBracket, upperBracket - curVal);
            const auto inc = pass0_increments(baseIncr, incrLimit, std::max(1, o.depth));
            const int use = o.depth >= 2 ? (int)inc.size() : 1;
            for (int j = 0; j < use; j++) {
                pts.push_back({curVal + inc[j], prev});
                prev = (int)pts.size() - 1;
                pts.push_back({curVal - inc[j], prev});
            }
            if ((rc = prefetch(pts))) return rc;
        }
        if (bump && (rc = evaluate(curVal, &curScore))) return rc;

        double lowerEval, higherEval, lowerEvalScore, higherEvalScore;
        double lastChange = 9999.9;
        double incr, diffDigits = 100.0;
        int lowBoundOvershoot = 0, upperBoundOvershoot = 0, positiveD2Num = 0, pass = 0;
        double incrLimit;
        bool limited = false;
        for (;;) {
            incrLimit = std::min(curVal - lowerBracket, upperBracket - curVal);
            incr = baseIncr;
            if (incr > incrLimit) {
                incr = incrLimit / 1.0001;
                limited = true;
            }
            higherEval = curVal + incr;
            if ((rc = evaluate(higherEval, &higherEvalScore))) return rc;
            // ADAPTIVE_BOUNDED_OPT: widen the increment until the score
            // difference is large enough for the finite differences
            bool cont = false;
            while (pass == 0 && !cont && !limited) {
                const double diff = std::fabs(curScore - higherEvalScore);
                if (diff != 0.0) diffDigits = std::log10(-curScore / diff);
                if (diffDigits > targetScoreDigits) {
                    baseIncr *= 5.0;
                    if (baseIncr > incrLimit) {
                        incr = incrLimit / 1.0001;
                        cont = true;
                    } else {
                        incr = baseIncr;
                    }
                    higherEval = curVal + incr;
                    if ((rc = evaluate(higherEval, &higherEvalScore))) return rc;
                } else {
                    cont = true;
                }
            }
            const double veryCloseToBound = baseIncr * 1.0001;
            const double closeToBound = baseIncr * 1.0002;
            lowerEval = curVal - incr;
            if ((rc = evaluate(lowerEval, &lowerEvalScore))) return rc;

            const double d11 = (higherEvalScore - curScore) / incr;
            const double d12 = (lowerEvalScore - curScore) / -incr;
            const double d1 = (d11 + d12) * 0.5;
            double d2 = (d11 - d12) / incr;
            const double est = -d1 / d2;
            double proposed = curVal + est;
            if (d11 - d12 == 0) d2 = 42.0;

            // the points straddle an optimum (or a minimum), or d1 is zero
            if ((d11 * d12 < 0.0) || (d1 == 0.0)) {
                if ((rc = check_score_and_restore(curScore, curVal, bestKnownScore, bestKnownVal, 0.0))) return rc;
                *result = o.lnL - initialScore;
                return GB_SUCCESS;
            }
            // positive second derivative: no Newton step, bump the value
            if (d2 > 0.0) {
                positiveD2Num++;
                double amtToBump;
                if (d1 > 0.0) {
                    if ((positiveD2Num + 1) % 3 == 0)
                        amtToBump = ((upperBracket + curVal) * 0.5) - curVal;
                    else
                        amtToBump = std::max(closeToBound, curVal * (0.02 * positiveD2Num));
                    proposed = curVal + amtToBump;
                } else {
                    if (positiveD2Num % 3 == 0 || (pass == 0 && boundBumped > 0.0))
                        amtToBump = curVal - (lowerBracket + veryCloseToBound);
                    else if ((positiveD2Num + 2) % 3 == 0)
                        amtToBump = curVal * (0.02 * positiveD2Num);
                    else
                        amtToBump = curVal - ((curVal + lowerBracket) * 0.5);
                    amtToBump = std::max(veryCloseToBound, amtToBump);
                    proposed = curVal - amtToBump;
                }
            }
            const double tolHere = pass > 0 ? 0.0 : kStepTol;
            if (d1 < 0.0 && proposed < lowerBracket + veryCloseToBound) {
                if (curVal - (lowerBracket + closeToBound) <= 0.0) {
                    if ((rc = check_score_and_restore(curScore, curVal, bestKnownScore, bestKnownVal, tolHere)))
                        return rc;
                    *result = o.lnL - initialScore;
                    return GB_SUCCESS;
                }
                lowBoundOvershoot++;
                if (lowBoundOvershoot == 2 || (lowBoundOvershoot == 1 && boundBumped > 0.0)) {
                    proposed = lowerBracket + veryCloseToBound;
                } else {
                    const double delta = std::max(veryCloseToBound, curVal - (curVal + lowerBracket) * 0.5);
                    proposed = curVal - delta;
                }
            } else if (d1 > 0.0 && proposed > upperBracket - veryCloseToBound) {
                if (upperBracket - closeToBound - curVal <= 0.0) {
                    if ((rc = check_score_and_restore(curScore, curVal, bestKnownScore, bestKnownVal, tolHere)))
                        return rc;
                    *result = o.lnL - initialScore;
                    return GB_SUCCESS;
                }
                upperBoundOvershoot++;
                if (upperBoundOvershoot == 2 || (upperBoundOvershoot == 1 && boundBumped > 0.0)) {
                    proposed = upperBracket - veryCloseToBound;
                } else {
                    const double delta = std::max(veryCloseToBound, (curVal + upperBracket) * 0.5 - curVal);
                    proposed = curVal + delta;
                }
            }
            double estImprove;
            if (d2 < 0.0)
                estImprove = d1 * (proposed - curVal) + (d2 * (proposed - curVal) * (proposed - curVal)) * 0.5;
            else
                estImprove = 9999.9;
            if (estImprove < optPrecision && curScore >= initialScore - 1.0e-6 && lastChange > -1.0e-6) {
                if ((rc = check_score_and_restore(curScore, curVal, bestKnownScore, bestKnownVal, tolHere))) return rc;
                *result = o.lnL - initialScore;
                return GB_SUCCESS;
            }
            if (pass > 1000) {
                if ((rc = check_score_and_restore(initialScore, initialVal, bestKnownScore, bestKnownVal, 0.0)))
                    return rc;
                *result = o.lnL - initialScore;
                return GB_SUCCESS;
            }
            if ((lowerBracket + closeToBound > proposed) && (upperBracket - closeToBound < proposed)) {
                if ((rc = check_score_and_restore(curScore, curVal, bestKnownScore, bestKnownVal, tolHere))) return rc;
                *result = o.lnL - initialScore;
                return GB_SUCCESS;
            }
            if (d1 <= 0.0 && curVal < upperBracket)
                upperBracket = curVal;
            else if (d1 > 0.0 && curVal > lowerBracket)
                lowerBracket = curVal;
            // the next pass's increment is fixed now: score the proposed value
            // and the next pair of points together
            if (o.depth >= 1) {
                const double lim = std::min(proposed - lowerBracket, upperBracket - proposed);
                const double nextIncr = baseIncr > lim ? lim / 1.0001 : baseIncr;
                if ((rc = prefetch({{proposed, -1}, {proposed + nextIncr, 0}, {proposed - nextIncr, 1}}))) return rc;
            }
            double proposedScore;
            if ((rc = evaluate(proposed, &proposedScore))) return rc;
            lastChange = proposedScore - curScore;
            curScore = proposedScore;
            curVal = proposed;
            pass++;
        }
    }
};

int optimize_bounded(Opt &o, int param, int which, double prec, double lowBound, double highBound,
                     double targetScoreDigits, double *improve) {
    if (!valid_param(o.m, param, which)) return GB_ERROR_OUT_OF_RANGE;
    Bounded b(o, param, which);
    return b.run(prec, get_param(o.m, param, which), lowBound, highBound, targetScoreDigits, improve);
}

// ---- the callers, with GARLI's bounds ----

// the model part of one BetterFinalOptimization pass (population.cpp:2690-2760)
int optimize_model(Opt &o, int mask, double prec, double *imp) {
    gb_model_params &m = o.m;
    for (int i = 0; i < 5; i++) imp[i] = 0.0;
    auto clamp = [](double v) { return (v < 0.0 && v > -1e-8) ? 0.0 : v; };
    double r;
    int rc;
    if ((mask & GB_OPT_OMEGA) && m.kind == GB_MODEL_CODON) {
        // Tree::OptimizeOmegaParameters, one omega class (tree.cpp:7186-7191)
        const double cur = m.omega;
        if ((rc = optimize_bounded(o, GB_PARAM_OMEGA, 0, prec, std::max(1.0e-5, cur / 5.0),
                                   std::max(std::min(9999.9, cur * 2.0), 0.01), 7.0, &r)))
            return rc;
        imp[GB_PARAM_OMEGA] += clamp(r);
    }
    if ((mask & GB_OPT_ALPHA) && m.categoryCount > 1 && m.kind != GB_MODEL_CODON) {
        const double a = m.alpha;
        if ((rc = optimize_bounded(o, GB_PARAM_ALPHA, 0, prec, std::min(0.05, a), std::max(999.9, a), 9.0, &r)))
            return rc;
        imp[GB_PARAM_ALPHA] += clamp(r);
    }
    if ((mask & GB_OPT_PINV) && m.hasPinv) {
        const double p = m.pinv;
        if ((rc = optimize_bounded(o, GB_PARAM_PINV, 0, prec, std::min(1.0e-8, p), m.maxPinv, 9.0, &r))) return rc;
        imp[GB_PARAM_PINV] += clamp(r);
    }
    if (mask & GB_OPT_FREQS) {
        // Tree::OptimizeEquilibriumFreqs (tree.cpp:7288-7305)
        const double maxChange = 1.2;
        double sum = 0.0;
        for (int i = 0; i < m.stateCount; i++) {
            const double cur = m.pi[i];
            if ((rc = optimize_bounded(o, GB_PARAM_STATE_FREQ, i, prec,
                                       std::min(std::max(m.stateCount > 4 ? 0.0001 : 0.01, cur / maxChange), cur),
                                       std::max(std::min(0.96, cur * maxChange), cur), 9.0, &r)))
                return rc;
            sum += r;
        }
        imp[GB_PARAM_STATE_FREQ] += clamp(sum);
    }
    if ((mask & GB_OPT_RATES) && m.kind != GB_MODEL_AMINO_ACID && m.nst > 1) {
        // Tree::OptimizeRelativeNucRates (tree.cpp:7307-7355)
        const double target = m.kind == GB_MODEL_CODON ? 7.0 : 9.0;
        const double maxChange = 5.0;
        double sum = 0.0;
        const int first = m.nst == 2 ? 1 : 0, last = m.nst == 2 ? 1 : 4;
        for (int i = first; i <= last; i++) {
            const double cur = m.rel[i];
            if ((rc = optimize_bounded(o, GB_PARAM_REL_RATE, i, prec, std::max(std::min(1.0e-3, cur), cur / maxChange),
                                       std::min(std::max(999.0, cur), cur * maxChange), target, &r)))
                return rc;
            sum += r;
        }
        imp[GB_PARAM_REL_RATE] += clamp(sum);
    }
    return GB_SUCCESS;
}

// Population::BetterFinalOptimization (population.cpp:2566-2790), one tree
int final_optimization(Opt &o, double branchOptPrecision, int mask, int maxPasses, double *out) {
    const double adapPrec = std::min(branchOptPrecision, 0.01);
    int rc, pass = 1;
    const long long evals0 = o.evals;
    int nnodes = 0;
    {
        int shape[5];
        if ((rc = gb_get_instance_shape(o.inst, shape))) return rc;
        nnodes = 2 * shape[0] - 2;
    }
    std::vector<double> blens(nnodes);
    bool goingToExit;
    do {
        const double precThisPass = std::max(adapPrec * std::pow(0.5, pass), 1e-10);
        const double paramPrecThisPass = std::max(precThisPass, 1e-5);
        if (fp_equals(o.lnL, -1.0, 1e-8) && (rc = score_current(o))) return rc;
        const double passStart = o.lnL;
        if ((rc = gbt_get_branch_lengths(o.tree, blens.data()))) return rc;
        double res[2];
        if ((rc = gbt_optimize_all_branches(o.tree, precThisPass, res))) return rc;
        if ((rc = score_current(o))) return rc;
        double trueImprove = o.lnL - passStart;
        if (trueImprove < 0.0) {
            // a pass that came out worse is undone (population.cpp:2638-2645)
            for (int nd = 1; nd < nnodes; nd++)
                if ((rc = gbt_set_branch_length(o.tree, nd, blens[nd]))) return rc;
            trueImprove = 0.0;
            if ((rc = score_current(o))) return rc;
        }
        double incr = trueImprove;
        double imp[5];
        if ((rc = optimize_model(o, mask, paramPrecThisPass, imp))) return rc;
        for (double v : imp) incr += v;
        goingToExit = !(incr > 1.0e-5 || precThisPass > 1.0e-4 || pass < 10);
        pass++;
    } while (!goingToExit && (maxPasses <= 0 || pass <= maxPasses));
    if ((rc = score_current(o))) return rc;
    out[0] = o.lnL;
    out[1] = pass - 1;
    out[2] = (double)(o.evals - evals0);
    return GB_SUCCESS;
}

}  // namespace

extern "C" {

int gbo_create(int tree, const gb_model_params *model, const double *aaExchangeabilities) {
    if (!model) return GB_ERROR_OUT_OF_RANGE;
    const int inst = gbt_get_instance(tree);
    if (inst < 0) return GB_ERROR_UNINITIALIZED_INSTANCE;
    int shape[5], cap[3];
    int rc;
    if ((rc = gb_get_instance_shape(inst, shape)) || (rc = gb_get_instance_capacity(inst, cap))) return rc;
    const gb_model_params &m = *model;
    if (m.stateCount != shape[2] || m.categoryCount != shape[3] || m.kind < 0 || m.kind > 2 ||
        (m.kind == GB_MODEL_AMINO_ACID && !aaExchangeabilities) || (m.kind != GB_MODEL_AMINO_ACID && m.nst != 1 &&
                                                                    m.nst != 2 && m.nst != 6))
        return GB_ERROR_OUT_OF_RANGE;
    const int ntax = shape[0], nint = ntax - 2, nnodes = 2 * ntax - 2;
    const int kmax = std::min({cap[2] - 1, (cap[0] - 3 * nint) / nint, cap[1] / nnodes - 1});
    if (kmax < 1) return GB_ERROR_OUT_OF_RANGE;  // room for at least one model besides the tree's
    auto *o = new Opt();
    o->tree = tree;
    o->inst = inst;
    o->kmax = kmax;
    // Speculation pays where a rescore costs little next to a call's fixed
    // latency (small trees); on large ones every model scored is HBM time, so
    // only the points known for certain are batched.
    o->depth = (long long)shape[4] * nint <= (1LL << 20) ? 4 : 1;
    if (m.kind == GB_MODEL_AMINO_ACID) o->exch.assign(aaExchangeabilities, aaExchangeabilities + 190);
    if ((rc = install(*o, m))) {
        delete o;
        return rc;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_opts.push_back(o);
    return (int)g_opts.size() - 1;
}

int gbo_destroy(int opt) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_opts[opt] = nullptr;
    }
    delete o;
    return GB_SUCCESS;
}

int gbo_get_model(int opt, gb_model_params *out) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    *out = o->m;
    return GB_SUCCESS;
}

int gbo_set_model(int opt, const gb_model_params *model) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!model || model->stateCount != o->m.stateCount || model->categoryCount != o->m.categoryCount ||
        model->kind != o->m.kind)
        return GB_ERROR_OUT_OF_RANGE;
    o->lnL = -1.0;
    return install(*o, *model);
}

int gbo_optimize_parameter(int opt, int param, int which, double precision, double lowBound, double highBound,
                           double targetScoreDigits, double *out) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!out || !(lowBound < highBound)) return GB_ERROR_OUT_OF_RANGE;
    double imp = 0.0;
    int rc = optimize_bounded(*o, param, which, precision, lowBound, highBound, targetScoreDigits, &imp);
    if (rc) return rc;
    out[0] = imp;
    out[1] = o->lnL;
    return GB_SUCCESS;
}

int gbo_optimize_model(int opt, int mask, double precision, double *out5) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!out5) return GB_ERROR_OUT_OF_RANGE;
    return optimize_model(*o, mask, precision, out5);
}

int gbo_final_optimization(int opt, double branchOptPrecision, int mask, int maxPasses, double *out3) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    if (!out3 || !(branchOptPrecision > 0.0)) return GB_ERROR_OUT_OF_RANGE;
    return final_optimization(*o, branchOptPrecision, mask, maxPasses, out3);
}

int gbo_set_batching(int opt, int on) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    o->depth = on < 0 ? 0 : on;
    return GB_SUCCESS;
}

int gbo_get_trace(int opt, double *values, double *scores, int capacity, double *initialScore) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    const int n = (int)o->traceVal.size();
    for (int i = 0; i < n && i < capacity; i++) {
        values[i] = o->traceVal[i];
        scores[i] = o->traceScore[i];
    }
    if (initialScore) *initialScore = o->traceInitial;
    return n;
}

int gbo_get_counters(int opt, long long *out3) {
    Opt *o = get(opt);
    if (!o) return GB_ERROR_UNINITIALIZED_INSTANCE;
    out3[0] = o->evals;
    out3[1] = o->scored;
    out3[2] = o->calls;
    return GB_SUCCESS;
}

}  // extern "C"
