"""Model-parameter optimisation on the device against the oracle (needs a B200).

Fixtures n.G4 / n.G5: 11 taxa x 2,178 sites, GTR+I+G4 / G5, GARLI's start trees
and printed parameters.

  * gbt_score_models: models scored together in one levelled pass give the
    scores the same models give one at a time through the tree's own CLAs;
  * gbo_optimize_parameter (Tree::OptimizeBoundedParameter) for alpha, pinv, a
    state frequency and a relative rate: every score it computed against the
    oracle's score of that model (1e-9 relative), its evaluations and result
    against oracle/modelopt.py replayed on those scores (exact), speculative
    batching on and off (identical);
  * gbo_final_optimization (Population::BetterFinalOptimization) on n.G4, n.G5
    and the codon fixture (GTR+I+G4/G5 with every parameter estimated; codons
    with six relative rates): the number the reference's scoring test compares
    with tests/data/expected.scr (allowed error 0.01 in tests/runtests.sh) to
    1e-4, and the oracle's final lnL to 1e-6.
"""
import numpy as np
import pytest

from conftest import fixture_params, load_fixture, scoring_setup, scoring_test_score
from garli_b200 import engine
from oracle import modelopt as mo
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

FIXTURES = ["z11x2178_nG4.json", "z11x2178_nG5.json"]


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if engine.lib().gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")


def _sides(name, kmax=8):
    fx, pd, c3, dl = load_fixture(name)
    fp = fixture_params(fx, pd)
    prm = engine.model_params(engine.MODEL_NUCLEOTIDE, fp["pi"], fp["rel"], fp["alpha"], fp["ncat"], fp["pinv"],
                              fp["max_pinv"])
    inst, tree, opt = engine.model_engine(pd, c3, dl, prm, kmax=kmax)
    P = mo.Params(mo.NUC, fp["pi"], fp["rel"], fp["alpha"], fp["ncat"], fp["pinv"], True, fp["max_pinv"])
    ot = orc.OracleTree(pd, c3, dl, mo.oracle_model(P))
    oopt = mo.ModelOptimizer(ot, P)
    return fx, pd, (inst, tree, opt), (ot, oopt)


def _close(*objs):
    for o in objs:
        o.close()


@pytest.mark.parametrize("name", FIXTURES)
def test_score_models_matches_one_at_a_time(name):
    fx, pd, (inst, tree, opt), (ot, _) = _sides(name)
    base = opt.params
    variants = []
    for a, p, r0 in ((0.4, 0.1, 1.0), (1.25, 0.30, 2.0), (3.0, 0.45, 0.7), (0.8, 0.2, 1.53)):
        m = engine.ModelParams.from_buffer_copy(base)
        m.alpha, m.pinv, m.rel[0] = a, p, r0
        variants.append(m)
    one = []
    for m in variants:
        opt.set_params(m)
        one.append(tree.score(0))
    # the same models in slots 1..4, scored together
    Qs, pis, bms = [], [], []
    for m in variants:
        Q, bm = engine.gtr_qmat(list(m.rel), np.array(m.pi[:4]))
        Qs.append(Q)
        pis.append(np.array(m.pi[:4]))
        bms.append(bm)
    inst.set_eigen_from_q([1, 2, 3, 4], np.array(Qs), np.array(pis), np.array(bms))
    for k, m in enumerate(variants):
        rates = engine.discrete_gamma(m.alpha, m.categoryCount)
        inst.set_model_slot(k + 1, np.array(m.pi[:4]), rates, np.full(m.categoryCount, (1 - m.pinv) / m.categoryCount),
                            m.pinv, True)
    together = tree.score_models([1, 2, 3, 4])
    for a, b in zip(one, together):
        assert abs(a - b) <= 1e-12 * abs(a), (one, together)
    # and against the oracle, model by model
    for m, g in zip(variants, together):
        P = mo.Params(mo.NUC, np.array(m.pi[:4]), np.array(m.rel[:]), m.alpha, m.categoryCount, m.pinv, True)
        ot.set_model(mo.oracle_model(P))
        ot.make_all_dirty()
        lo = ot.score(0)
        assert abs(g - lo) <= 1e-9 * abs(lo), (g, lo)
    _close(opt, tree, inst, ot)


CASES = [
    ("alpha", engine.PARAM_ALPHA, mo.ALPHA, 0),
    ("pinv", engine.PARAM_PINV, mo.PINV, 0),
    ("freq2", engine.PARAM_STATE_FREQ, mo.FREQ, 2),
    ("rate1", engine.PARAM_REL_RATE, mo.REL, 1),
]


def _bounds(param, cur, max_pinv):
    """GARLI's bounds for each optimised parameter (population.cpp:2702, :2727; tree.cpp:7296-7299, :7351-7354)."""
    if param == mo.ALPHA:
        return min(0.05, cur), max(999.9, cur)
    if param == mo.PINV:
        return min(1.0e-8, cur), max_pinv
    if param == mo.FREQ:
        return min(max(0.01, cur / 1.2), cur), max(min(0.96, cur * 1.2), cur)
    return max(min(1.0e-3, cur), cur / 5.0), min(max(999.0, cur), cur * 5.0)


def _start(opt, oopt, oparam, m_init):
    """The fixture's model, with alpha and pinv away from the optimum so that
    the optimiser takes several passes."""
    m = engine.ModelParams.from_buffer_copy(m_init)
    if oparam == mo.ALPHA:
        m.alpha = oopt.p.alpha = 0.6
    elif oparam == mo.PINV:
        m.pinv = oopt.p.pinv = 0.15
    opt.set_params(m)
    return m


@pytest.mark.parametrize("name", FIXTURES[:1])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_optimize_parameter_matches_oracle(name, case):
    """Two checks that together cover OptimizeBoundedParameter on the device:
    every score it computed equals the oracle's score of that model (1e-9
    relative), and the oracle's restatement of the optimiser, fed those scores,
    makes the same evaluations and ends on the same value and lnL, bit for bit.
    (The optimiser's finite differences over increments of 1e-6 .. 1e-4 turn
    1e-12 score differences into different proposals, so two independent FP64
    runs agree only to about the requested precision; the replay checks the
    decisions exactly.)  Speculative batching changes nothing."""
    _, gparam, oparam, which = case
    fx, pd, (inst, tree, opt), (ot, oopt) = _sides(name)
    m_init = engine.ModelParams.from_buffer_copy(opt.params)
    runs = {}
    for depth in (3, 0):
        _start(opt, oopt, oparam, m_init)
        start_p = mo.Params(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in vars(oopt.p).items()})
        cur = mo.get_param(start_p, oparam, which)
        lo, hi = _bounds(oparam, cur, start_p.max_pinv)
        opt.set_batching(depth)
        c0 = opt.counters()
        gi, gl = opt.optimize_parameter(gparam, which, 0.005, lo, hi)
        c1 = opt.counters()
        ini, vals, scores = opt.trace()
        gm = opt.params
        gv = {mo.ALPHA: gm.alpha, mo.PINV: gm.pinv, mo.FREQ: gm.pi[which], mo.REL: gm.rel[which]}[oparam]
        runs[depth] = dict(gl=gl, gv=gv, ini=ini, vals=vals.copy(), scores=scores.copy(), lo=lo, hi=hi,
                           calls=c1["score_calls"] - c0["score_calls"], evals=c1["evaluations"] - c0["evaluations"])
        assert abs(tree.score(0) - gl) <= 1e-9 * abs(gl)
    a, b = runs[3], runs[0]
    assert np.array_equal(a["vals"], b["vals"]) and a["gv"] == b["gv"], (a, b)
    assert np.allclose(a["scores"], b["scores"], rtol=1e-13, atol=0.0)
    assert a["evals"] == b["evals"] == len(a["vals"]) and b["calls"] == b["evals"] and a["calls"] < a["evals"]
    # every score against the oracle, models built along GARLI's chain of setter calls
    P = mo.Params(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in vars(start_p).items()})
    for v, sc in zip(a["vals"], a["scores"]):
        mo.set_param(P, oparam, which, float(v))
        ot.set_model(mo.oracle_model(P))
        ot.make_all_dirty()
        lo_ = ot.score(0)
        assert abs(sc - lo_) <= 1e-9 * abs(lo_), (v, sc, lo_)
    # the oracle's optimiser replayed on the device's scores
    oopt.p = mo.Params(**{k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in vars(start_p).items()})
    oopt.lnL = a["ini"]
    oopt.replay = list(zip(a["vals"].tolist(), a["scores"].tolist()))
    oopt.evals = 0
    oi = oopt.optimize_bounded(oparam, which, 0.005, a["lo"], a["hi"])
    assert oopt.replay == [] and oopt.evals == len(a["vals"])
    assert mo.get_param(oopt.p, oparam, which) == a["gv"], (mo.get_param(oopt.p, oparam, which), a["gv"])
    assert oopt.lnL == a["gl"]
    _close(opt, tree, inst, ot)


def _scoring_sides(name, kmax=8):
    fx, pd, c3, dl = load_fixture(name)
    sp = scoring_setup(fx, pd)
    prm = engine.model_params(sp["kind"], sp["pi"], sp["rel"], sp["alpha"], sp["ncat"], sp["pinv"], sp["max_pinv"],
                              sp["omega"])
    inst, tree, opt = engine.model_engine(pd, c3, dl, prm, kmax=kmax)
    P = mo.Params(sp["kind"], sp["pi"], sp["rel"], sp["alpha"], sp["ncat"], sp["pinv"] or 0.0,
                  sp["pinv"] is not None, sp["max_pinv"], sp["omega"])
    ot = orc.OracleTree(pd, c3, dl, mo.oracle_model(P))
    oopt = mo.ModelOptimizer(ot, P)
    return fx, pd, sp, (inst, tree, opt), (ot, oopt)


@pytest.mark.parametrize("name", FIXTURES + ["z11x2178_codon.json"])
def test_final_optimization_reproduces_expected_scr(name):
    fx, pd, sp, (inst, tree, opt), (ot, oopt) = _scoring_sides(name)
    gl, gpasses, gevals = opt.final_optimization(0.01, sp["mask"])
    tree.make_all_dirty()
    assert abs(tree.score(0) - gl) <= 1e-9 * abs(gl)
    scr = scoring_test_score(fx, gl, inst.site_lnl())
    assert abs(scr - fx["scoring_test"]["expected_scr"]) < 1e-4, (scr, fx["scoring_test"])
    ol, opasses, oevals = oopt.final_optimization(0.01, sp["mask"])
    assert abs(gl - ol) <= 1e-6, (gl, ol)
    assert gpasses == opasses
    _close(opt, tree, inst, ot)
