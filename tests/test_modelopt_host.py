"""The model optimiser's host logic (gb_modelopt.cpp) on CPU, against a fake engine.

gb_modelopt.cpp is compiled with the real host model math (gb_model.cpp) and
tests/host_fake/fake_engine.cpp, a fake of the engine calls it makes that
scores each model slot on a smooth surface.  Checked without a GPU:
  * OptimizeBoundedParameter for alpha, pinv, a state frequency and a relative
    rate: the oracle's restatement (oracle/modelopt.py), replayed on the
    evaluations the C++ recorded, makes the same evaluations and ends on the
    same value and lnL, bit for bit;
  * batching (speculative depths 1 and 4) changes no evaluation and no result,
    and takes fewer score calls than evaluations;
  * BetterFinalOptimization ends on the same model at every batching depth;
  * argument errors come back as GB_ERROR_* codes.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from garli_b200 import engine
from oracle import modelopt as mo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def fake(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("fake") / "libgbo_fake.so")
    srcs = [os.path.join(ROOT, "garli_b200", "csrc", "gb_modelopt.cpp"),
            os.path.join(ROOT, "garli_b200", "csrc", "gb_model.cpp"),
            os.path.join(ROOT, "tests", "host_fake", "fake_engine.cpp")]
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", os.path.join(ROOT, "include")] + srcs +
                   ["-o", out], check=True)
    L = C.CDLL(out)
    for n, (r, a) in engine.SIGNATURES.items():
        if n.startswith("gbo_"):
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
    L.fake_counters.argtypes = [C.POINTER(C.c_longlong)]
    return L


START = dict(pi=[0.25, 0.24, 0.26, 0.25], rel=[1.2, 3.0, 1.9, 1.1, 4.0, 1.0], alpha=0.6, ncat=4, pinv=0.15,
             max_pinv=0.49)


def _params():
    return engine.model_params(engine.MODEL_NUCLEOTIDE, START["pi"], START["rel"], START["alpha"], START["ncat"],
                               START["pinv"], START["max_pinv"])


def _opt_params():
    return mo.Params(mo.NUC, np.array(START["pi"]), np.array(START["rel"]), START["alpha"], START["ncat"],
                     START["pinv"], True, START["max_pinv"])


def _calls(L):
    c = (C.c_longlong * 2)()
    L.fake_counters(c)
    return c[0], c[1]


def _trace(L, h):
    ini = C.c_double()
    n = L.gbo_get_trace(h, None, None, 0, C.byref(ini))
    v, s = np.zeros(max(n, 1)), np.zeros(max(n, 1))
    L.gbo_get_trace(h, v.ctypes.data_as(C.POINTER(C.c_double)), s.ctypes.data_as(C.POINTER(C.c_double)), n, None)
    return ini.value, v[:n], s[:n]


CASES = [(engine.PARAM_ALPHA, mo.ALPHA, 0), (engine.PARAM_PINV, mo.PINV, 0), (engine.PARAM_STATE_FREQ, mo.FREQ, 2),
         (engine.PARAM_REL_RATE, mo.REL, 1)]


def _bounds(param, cur, max_pinv):
    if param == mo.ALPHA:
        return min(0.05, cur), max(999.9, cur)
    if param == mo.PINV:
        return min(1.0e-8, cur), max_pinv
    if param == mo.FREQ:
        return min(max(0.01, cur / 1.2), cur), max(min(0.96, cur * 1.2), cur)
    return max(min(1.0e-3, cur), cur / 5.0), min(max(999.0, cur), cur * 5.0)


@pytest.mark.parametrize("case", CASES, ids=["alpha", "pinv", "freq2", "rate1"])
def test_bounded_optimiser_matches_restatement(fake, case):
    gparam, oparam, which = case
    P = _opt_params()
    cur = mo.get_param(P, oparam, which)
    lo, hi = _bounds(oparam, cur, P.max_pinv)
    runs = {}
    for depth in (0, 1, 4):
        m = _params()
        h = fake.gbo_create(0, C.byref(m), None)
        assert h >= 0
        assert fake.gbo_set_batching(h, depth) == 0
        c0 = _calls(fake)
        out = np.zeros(2)
        assert fake.gbo_optimize_parameter(h, gparam, which, 0.005, lo, hi, 9.0,
                                           out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        c1 = _calls(fake)
        ini, vals, scores = _trace(fake, h)
        got = engine.ModelParams()
        fake.gbo_get_model(h, C.byref(got))
        gv = {mo.ALPHA: got.alpha, mo.PINV: got.pinv, mo.FREQ: got.pi[which], mo.REL: got.rel[which]}[oparam]
        runs[depth] = (out.copy(), ini, vals, scores, gv, c1[0] - c0[0], len(vals))
        fake.gbo_destroy(h)
    ref = runs[0]
    assert len(ref[2]) > 4
    for depth in (1, 4):
        r = runs[depth]
        assert np.array_equal(r[2], ref[2]) and np.array_equal(r[3], ref[3]) and r[4] == ref[4], depth
        assert r[5] < r[6], (depth, r[5], r[6])  # fewer score calls than evaluations
    assert ref[5] == ref[6]
    # the restatement replayed on the recorded evaluations
    o = mo.ModelOptimizer(None, P)
    o.lnL = ref[1]
    o.replay = list(zip(ref[2].tolist(), ref[3].tolist()))
    imp = o.optimize_bounded(oparam, which, 0.005, lo, hi)
    assert o.replay == [] and o.evals == len(ref[2])
    assert mo.get_param(o.p, oparam, which) == ref[4]
    assert o.lnL == ref[0][1] and imp == ref[0][0]


def test_final_optimization_same_at_every_depth(fake):
    ends = []
    for depth in (0, 1, 4):
        m = _params()
        h = fake.gbo_create(0, C.byref(m), None)
        fake.gbo_set_batching(h, depth)
        out = np.zeros(3)
        assert fake.gbo_final_optimization(h, 0.01, 15, 0, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        got = engine.ModelParams()
        fake.gbo_get_model(h, C.byref(got))
        ends.append((out[0], out[1], out[2], got.alpha, got.pinv, tuple(got.pi[:4]), tuple(got.rel[:6])))
        fake.gbo_destroy(h)
    assert ends[0][1] >= 10 and ends[0][2] > 100  # GARLI's exit rule: at least 10 passes
    assert ends[0] == ends[1] == ends[2]
    # the surface's optimum: alpha 1.25, pinv 0.3
    assert abs(ends[0][3] - 1.25) < 0.02 and abs(ends[0][4] - 0.3) < 0.01


def test_argument_errors(fake):
    m = _params()
    assert fake.gbo_create(7, C.byref(m), None) == engine.GB_ERROR_UNINITIALIZED_INSTANCE
    bad = _params()
    bad.categoryCount = 3  # not the instance's
    assert fake.gbo_create(0, C.byref(bad), None) == engine.GB_ERROR_OUT_OF_RANGE
    h = fake.gbo_create(0, C.byref(m), None)
    out = np.zeros(2)
    op = out.ctypes.data_as(C.POINTER(C.c_double))
    assert fake.gbo_optimize_parameter(h, engine.PARAM_OMEGA, 0, 0.01, 0.1, 2.0, 9.0, op) == engine.GB_ERROR_OUT_OF_RANGE
    assert fake.gbo_optimize_parameter(h, engine.PARAM_REL_RATE, 5, 0.01, 0.1, 2.0, 9.0, op) == engine.GB_ERROR_OUT_OF_RANGE
    assert fake.gbo_optimize_parameter(h, engine.PARAM_ALPHA, 0, 0.01, 2.0, 1.0, 9.0, op) == engine.GB_ERROR_OUT_OF_RANGE
    fake.gbo_destroy(h)
    assert fake.gbo_optimize_parameter(h, engine.PARAM_ALPHA, 0, 0.01, 0.1, 2.0, 9.0, op) == \
        engine.GB_ERROR_UNINITIALIZED_INSTANCE
