"""CPU restatement of GARLI's model-parameter optimisation, on the oracle tree.

TEST INFRASTRUCTURE ONLY (the checker of gbo_* in the engine); the garli_b200
package never imports it.

Follows, one evaluation at a time in GARLI's order:
  * Model setters: SetAlpha (model.h:1742, DiscreteGamma model.cpp:2170-2201),
    SetPinv (model.h:1733), SetEquilibriumFreq (model.h:1501-1516) with
    NormalizeSumConstrainedValues (model.h:1681-1731), SetRelativeNucRate
    (model.h:1518-1531), SetOmega (model.h:1797);
  * Tree::SetAndEvaluateParameter (optimization.cpp:244-268),
    CheckScoreAndRestore (:271-301) and OptimizeBoundedParameter (:332-776)
    with NEW_BUMPING and ADAPTIVE_BOUNDED_OPT (defs.h:63-67), double precision
    (STEP_TOL 1e-8, optimization.cpp:33-39);
  * OptimizeEquilibriumFreqs (tree.cpp:7288-7305), OptimizeRelativeNucRates
    (tree.cpp:7307-7355), one-class omega (tree.cpp:7186-7191), alpha and pinv
    bounds (population.cpp:2702, :2727);
  * Population::BetterFinalOptimization (population.cpp:2566-2790).
Each model is built with the oracle's own Q, eigen and discrete-gamma code.
"""
from __future__ import annotations

import copy
import math
from dataclasses import dataclass, field

import numpy as np

from . import oracle as orc

STEP_TOL = 1.0e-8
FP_EPS = 2.220446049250313e-16

ALPHA, PINV, FREQ, REL, OMEGA = 0, 1, 2, 3, 4
NUC, AA, CODON = 0, 1, 2


@dataclass
class Params:
    kind: int
    pi: np.ndarray
    rel: np.ndarray = field(default_factory=lambda: np.ones(6))
    alpha: float = 0.5
    ncat: int = 1
    pinv: float = 0.0
    has_pinv: bool = False
    max_pinv: float = 0.0
    omega: float = 1.0
    nst: int = 6


@dataclass
class _OracleModel:
    eval_scaled: np.ndarray
    U: np.ndarray
    Uinv: np.ndarray
    pi: np.ndarray
    rates: np.ndarray
    probs: np.ndarray
    pinv: float
    has_pinv: bool
    ncat: int


def oracle_model(p: Params, exch=None) -> _OracleModel:
    """The oracle-side model of parameters p (Model::UpdateQMat, CalcEigenStuff, DiscreteGamma)."""
    if p.kind == NUC:
        Q, bm = orc.gtr_qmat(p.rel, p.pi)
    elif p.kind == AA:
        Q, bm = orc.aa_qmat(exch, p.pi)
    else:
        Q, bm = orc.codon_qmat6(p.rel, p.omega, p.pi)
    ev, U, Ui = orc.eigen(Q, p.pi)
    rates = orc.discrete_gamma(p.alpha, p.ncat) if p.ncat > 1 else np.ones(1)
    pinv = p.pinv if p.has_pinv else 0.0
    probs = np.full(p.ncat, (1.0 - pinv) / p.ncat)
    return _OracleModel(ev * bm, U, Ui, np.array(p.pi, dtype=np.float64), rates, probs, pinv, p.has_pinv, p.ncat)


def normalize_sum_constrained(vals, target, min_val, to_not_change):
    """Model::NormalizeSumConstrainedValues (model.h:1681-1731), in place."""
    n = len(vals)
    some_min = False
    min_sum = 0.0
    s = 0.0
    for i in range(n):
        if i != to_not_change:
            s += vals[i]
            if vals[i] < min_val:
                some_min = True
    if some_min or not abs(s - target) < min_val * 0.01:
        while True:
            unfixed = target - (0.0 if to_not_change < 0 else vals[to_not_change]) - min_sum
            rescale = unfixed / s
            some_min = False
            s = 0.0
            for i in range(n):
                if i != to_not_change and vals[i] > 0.0:
                    vals[i] *= rescale
                    if vals[i] < min_val:
                        vals[i] = -1.0
                        min_sum += min_val
                        some_min = True
                    else:
                        s += vals[i]
            if not some_min:
                break
    for i in range(n):
        if vals[i] < 0.0:
            vals[i] = min_val


def set_param(p: Params, param: int, which: int, val: float):
    if param == ALPHA:
        p.alpha = val
    elif param == PINV:
        p.pinv = val
    elif param == FREQ:
        p.pi[which] = val
        normalize_sum_constrained(p.pi, 1.0, 1e-4, which)
    elif param == REL:
        if p.nst == 2:
            # AG and CT share the transition rate, the rest the transversion rate
            group = (1, 4) if which in (1, 4) else (0, 2, 3, 5)
            for i in group:
                p.rel[i] = val
        else:
            p.rel[which] = val
        if not abs(p.rel[5] - 1.0) < 1.0e-12:
            sc = 1.0 / p.rel[5]
            for i in range(5):
                p.rel[i] *= sc
            p.rel[5] *= sc
    elif param == OMEGA:
        p.omega = val


def get_param(p: Params, param: int, which: int) -> float:
    if param == ALPHA:
        return p.alpha
    if param == PINV:
        return p.pinv
    if param == OMEGA:
        return p.omega
    return float(p.pi[which] if param == FREQ else p.rel[which])


class ModelOptimizer:
    """GARLI's model optimisation of one oracle tree."""

    def __init__(self, otree: "orc.OracleTree", params: Params, exch=None):
        self.ot = otree
        self.p = copy.deepcopy(params)
        self.p.pi = np.array(self.p.pi, dtype=np.float64)
        self.p.rel = np.array(self.p.rel, dtype=np.float64)
        self.exch = exch
        self.lnL = -1.0
        self.evals = 0
        # replay: scores taken, in order, from a recorded sequence of
        # (value, score) instead of the oracle tree (checks the decisions alone)
        self.replay = None
        self._install()

    def _install(self):
        if self.ot is None:  # replay only: no tree
            return
        self.ot.set_model(oracle_model(self.p, self.exch))
        self.ot.make_all_dirty()

    def score(self):
        self.lnL = self.ot.score(0)
        return self.lnL

    # Tree::SetAndEvaluateParameter (optimization.cpp:244-268)
    def _set_and_evaluate(self, param, which, val, best):
        set_param(self.p, param, which, val)
        if self.replay is not None:
            rv, rs = self.replay.pop(0)
            if rv != val:
                raise AssertionError(f"evaluation {self.evals}: value {val!r}, recorded {rv!r}")
            self.lnL = rs
        else:
            self._install()
            self.score()
        self.evals += 1
        if self.lnL > best[0]:
            best[1] = val
            best[0] = self.lnL
        return self.lnL

    # Tree::CheckScoreAndRestore (optimization.cpp:271-301)
    def _check_score_and_restore(self, param, which, other_score, other_val, best_score, best_val, tol):
        if other_score + tol < best_score:
            set_param(self.p, param, which, best_val)
            other_score = best_score
        else:
            set_param(self.p, param, which, other_val)
        if self.replay is None:
            self._install()
        self.lnL = other_score

    # Tree::OptimizeBoundedParameter (optimization.cpp:332-776)
    def optimize_bounded(self, param, which, opt_precision, low_bound, high_bound, target_digits=9.0):
        initial_val = get_param(self.p, param, which)
        if abs(self.lnL - (-1.0)) < max(1.0e-8, FP_EPS * 2.0):
            self.score()
        base_incr = min(max(0.001 * opt_precision, 1.0e-6), initial_val * 0.01)
        cur_val = initial_val
        initial_score = cur_score = self.lnL
        best = [initial_score, initial_val]  # bestKnownScore, bestKnownVal

        def done(other_score, other_val, tol):
            self._check_score_and_restore(param, which, other_score, other_val, best[0], best[1], tol)
            return self.lnL - initial_score

        # NEW_BUMPING
        required_window = (base_incr * 1.0001) * 2.0
        actual_window = high_bound - low_bound
        if actual_window < required_window:
            return 0.0
        bound_bumped = -1.0
        bump_amt = base_incr * 25.0001
        if low_bound + bump_amt > initial_val:
            if low_bound + bump_amt > high_bound - bump_amt:
                bump_amt = actual_window / 2.0
            bound_bumped = abs(cur_val - (low_bound + bump_amt))
            cur_val = low_bound + bump_amt
            cur_score = self._set_and_evaluate(param, which, cur_val, best)
        elif high_bound - bump_amt < initial_val:
            if high_bound - bump_amt < low_bound + bump_amt:
                bump_amt = actual_window / 2.0
            cur_val = high_bound - bump_amt
            bound_bumped = initial_val - cur_val
            cur_score = self._set_and_evaluate(param, which, cur_val, best)

        last_change = 9999.9
        upper_bracket, lower_bracket = high_bound, low_bound
        diff_digits = 100.0
        low_overshoot = up_overshoot = 0
        pos_d2 = 0
        npass = 0
        limited = False
        while True:
            incr_limit = min(cur_val - lower_bracket, upper_bracket - cur_val)
            incr = base_incr
            if incr > incr_limit:
                incr = incr_limit / 1.0001
                limited = True
            higher_eval = cur_val + incr
            higher_score = self._set_and_evaluate(param, which, higher_eval, best)
            cont = False
            while npass == 0 and not cont and not limited:
                diff = abs(cur_score - higher_score)
                if diff != 0.0:
                    diff_digits = math.log10(-cur_score / diff)
                if diff_digits > target_digits:
                    base_incr *= 5.0
                    if base_incr > incr_limit:
                        incr = incr_limit / 1.0001
                        cont = True
                    else:
                        incr = base_incr
                    higher_eval = cur_val + incr
                    higher_score = self._set_and_evaluate(param, which, higher_eval, best)
                else:
                    cont = True
            very_close = base_incr * 1.0001
            close = base_incr * 1.0002
            lower_eval = cur_val - incr
            lower_score = self._set_and_evaluate(param, which, lower_eval, best)

            d11 = (higher_score - cur_score) / incr
            d12 = (lower_score - cur_score) / -incr
            d1 = (d11 + d12) * 0.5
            d2 = (d11 - d12) / incr
            with np.errstate(divide="ignore", invalid="ignore"):
                est = -d1 / d2 if d2 != 0.0 else (math.copysign(math.inf, -d1) if d1 != 0.0 else math.nan)
            proposed = cur_val + est
            if d11 - d12 == 0:
                d2 = 42.0
            if d11 * d12 < 0.0 or d1 == 0.0:
                return done(cur_score, cur_val, 0.0)
            if d2 > 0.0:
                pos_d2 += 1
                if d1 > 0.0:
                    if (pos_d2 + 1) % 3 == 0:
                        amt = ((upper_bracket + cur_val) * 0.5) - cur_val
                    else:
                        amt = max(close, cur_val * (0.02 * pos_d2))
                    proposed = cur_val + amt
                else:
                    if pos_d2 % 3 == 0 or (npass == 0 and bound_bumped > 0.0):
                        amt = cur_val - (lower_bracket + very_close)
                    elif (pos_d2 + 2) % 3 == 0:
                        amt = cur_val * (0.02 * pos_d2)
                    else:
                        amt = cur_val - ((cur_val + lower_bracket) * 0.5)
                    amt = max(very_close, amt)
                    proposed = cur_val - amt
            tol = 0.0 if npass > 0 else STEP_TOL
            if d1 < 0.0 and proposed < lower_bracket + very_close:
                if cur_val - (lower_bracket + close) <= 0.0:
                    return done(cur_score, cur_val, tol)
                low_overshoot += 1
                if low_overshoot == 2 or (low_overshoot == 1 and bound_bumped > 0.0):
                    proposed = lower_bracket + very_close
                else:
                    delta = max(very_close, cur_val - (cur_val + lower_bracket) * 0.5)
                    proposed = cur_val - delta
            elif d1 > 0.0 and proposed > upper_bracket - very_close:
                if upper_bracket - close - cur_val <= 0.0:
                    return done(cur_score, cur_val, tol)
                up_overshoot += 1
                if up_overshoot == 2 or (up_overshoot == 1 and bound_bumped > 0.0):
                    proposed = upper_bracket - very_close
                else:
                    delta = max(very_close, (cur_val + upper_bracket) * 0.5 - cur_val)
                    proposed = cur_val + delta
            if d2 < 0.0:
                est_improve = d1 * (proposed - cur_val) + (d2 * (proposed - cur_val) * (proposed - cur_val)) * 0.5
            else:
                est_improve = 9999.9
            if est_improve < opt_precision and cur_score >= initial_score - 1.0e-6 and last_change > -1.0e-6:
                return done(cur_score, cur_val, tol)
            if npass > 1000:
                return done(initial_score, initial_val, 0.0)
            if lower_bracket + close > proposed and upper_bracket - close < proposed:
                return done(cur_score, cur_val, tol)
            if d1 <= 0.0 and cur_val < upper_bracket:
                upper_bracket = cur_val
            elif d1 > 0.0 and cur_val > lower_bracket:
                lower_bracket = cur_val
            prop_score = self._set_and_evaluate(param, which, proposed, best)
            last_change = prop_score - cur_score
            cur_score = prop_score
            cur_val = proposed
            npass += 1

    def optimize_model(self, mask, prec):
        """The model part of one BetterFinalOptimization pass (population.cpp:2690-2760)."""
        p = self.p
        imp = np.zeros(5)

        def clamp(v):
            return 0.0 if -1e-8 < v < 0.0 else v

        if mask & 16 and p.kind == CODON:
            cur = p.omega
            imp[OMEGA] += clamp(self.optimize_bounded(OMEGA, 0, prec, max(1.0e-5, cur / 5.0),
                                                      max(min(9999.9, cur * 2.0), 0.01), 7.0))
        if mask & 1 and p.ncat > 1 and p.kind != CODON:
            a = p.alpha
            imp[ALPHA] += clamp(self.optimize_bounded(ALPHA, 0, prec, min(0.05, a), max(999.9, a)))
        if mask & 2 and p.has_pinv:
            pv = p.pinv
            imp[PINV] += clamp(self.optimize_bounded(PINV, 0, prec, min(1.0e-8, pv), p.max_pinv))
        if mask & 4:
            s = 0.0
            for i in range(len(p.pi)):
                cur = p.pi[i]
                lo = min(max(0.0001 if len(p.pi) > 4 else 0.01, cur / 1.2), cur)
                hi = max(min(0.96, cur * 1.2), cur)
                s += self.optimize_bounded(FREQ, i, prec, lo, hi)
            imp[FREQ] += clamp(s)
        if mask & 8 and p.kind != AA and p.nst > 1:
            target = 7.0 if p.kind == CODON else 9.0
            s = 0.0
            for i in ([1] if p.nst == 2 else range(5)):
                cur = p.rel[i]
                s += self.optimize_bounded(REL, i, prec, max(min(1.0e-3, cur), cur / 5.0),
                                           min(max(999.0, cur), cur * 5.0), target)
            imp[REL] += clamp(s)
        return imp

    def final_optimization(self, branch_precision=0.01, mask=31, max_passes=0):
        """Population::BetterFinalOptimization (population.cpp:2566-2790) for one tree."""
        adap = min(branch_precision, 0.01)
        npass = 1
        ev0 = self.evals
        while True:
            prec = max(adap * 0.5 ** npass, 1e-10)
            pprec = max(prec, 1e-5)
            if abs(self.lnL + 1.0) < 1e-8:
                self.score()
            start = self.lnL
            blens = self.ot.branch_lengths()
            self.ot.optimize_all_branches(prec)
            self.score()
            true_improve = self.lnL - start
            if true_improve < 0.0:
                for nd in range(1, len(blens)):
                    self.ot.set_branch_length(nd, blens[nd])
                true_improve = 0.0
                self.score()
            incr = true_improve + float(self.optimize_model(mask, pprec).sum())
            going = not (incr > 1.0e-5 or prec > 1.0e-4 or npass < 10)
            npass += 1
            if going or (max_passes > 0 and npass > max_passes):
                break
        self.score()
        return self.lnL, npass - 1, self.evals - ev0
