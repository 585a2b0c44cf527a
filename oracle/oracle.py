"""ctypes wrapper of the CPU oracle (oracle/garli_oracle.c).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the cpu_baseline
leg of bench.py use this module as the checker (and the CPU timing baseline);
the garli_b200 package never imports it.

Two builds exist: ``liboracle.so`` (strict IEEE order, no fused multiply-add;
the parity reference) and ``liboracle_fast.so`` (GARLI's own -O3 -ffast-math
flags, configure.ac:217; the timed CPU baseline).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict[str, C.CDLL] = {}
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_U8 = C.POINTER(C.c_ubyte)

SIGS = {
    "or_gtr_qmat": (None, [_D, _D, _D, _D]),
    "or_aa_qmat": (None, [_D, _D, _D, _D]),
    "or_codon_qmat": (C.c_int, [C.c_double, C.c_double, _D, _D, _D]),
    "or_codon_qmat6": (C.c_int, [_D, C.c_double, _D, _D, _D]),
    "or_eigen": (C.c_int, [C.c_int, _D, _D, _D, _D, _D]),
    "or_discrete_gamma": (None, [C.c_double, C.c_int, _D]),
    "or_pmats": (None, [C.c_int, C.c_int, _D, _D, _D, _D, C.c_double, C.c_int, C.c_double, _D, _D, _D]),
    "or_tree_new": (C.c_void_p, [C.c_int, C.c_int, C.c_int, C.c_int, _I, _D, _U8, _I, C.c_int, _I]),
    "or_tree_free": (None, [C.c_void_p]),
    "or_tree_set_model": (None, [C.c_void_p, _D, _D, _D, _D, _D, _D, C.c_double, C.c_int]),
    "or_tree_set_rescale_every": (None, [C.c_void_p, C.c_int]),
    "or_tree_get_rescale_every": (C.c_int, [C.c_void_p]),
    "or_tree_score": (C.c_double, [C.c_void_p, C.c_int]),
    "or_tree_derivs": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "or_tree_nr_optimize": (C.c_double, [C.c_void_p, C.c_double, C.c_int]),
    "or_tree_optimize_all": (C.c_double, [C.c_void_p, C.c_double]),
    "or_tree_set_blen": (None, [C.c_void_p, C.c_int, C.c_double]),
    "or_tree_get_blen": (C.c_double, [C.c_void_p, C.c_int]),
    "or_tree_dirty_all": (None, [C.c_void_p]),
    "or_tree_lnl": (C.c_double, [C.c_void_p]),
    "or_tree_get_cla": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _I]),
    "or_tree_cla_rank": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "or_tree_cla_dirty": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "or_tree_site_lnl": (C.c_int, [C.c_void_p, _D]),
    "or_tree_cla_count": (C.c_long, [C.c_void_p]),
    "or_tree_deriv_count": (C.c_long, [C.c_void_p]),
    "or_set_threads": (None, [C.c_int]),
    "or_get_threads": (C.c_int, []),
    "or_rescale_tables": (None, [_I, _D, _D]),
}


def build():
    """Compile both oracle builds with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(fast: bool = False) -> C.CDLL:
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name not in _LIBS:
        path = os.path.join(HERE, name)
        src = os.path.join(HERE, "garli_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = C.CDLL(path)
        for n, (res, args) in SIGS.items():
            f = getattr(L, n)
            f.restype = res
            f.argtypes = args
        _LIBS[name] = L
    return _LIBS[name]


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def gtr_qmat(rel, pi):
    Q = np.zeros((4, 4)); bm = C.c_double()
    lib().or_gtr_qmat(_p(_f(rel), C.c_double), _p(_f(pi), C.c_double), _p(Q, C.c_double), C.byref(bm))
    return Q, bm.value


def aa_qmat(exch, pi):
    Q = np.zeros((20, 20)); bm = C.c_double()
    lib().or_aa_qmat(_p(_f(exch), C.c_double), _p(_f(pi), C.c_double), _p(Q, C.c_double), C.byref(bm))
    return Q, bm.value


def codon_qmat(kappa, omega, pi):
    Q = np.zeros((61, 61)); bm = C.c_double()
    lib().or_codon_qmat(kappa, omega, _p(_f(pi), C.c_double), _p(Q, C.c_double), C.byref(bm))
    return Q, bm.value


def codon_qmat6(rel6, omega, pi):
    Q = np.zeros((61, 61)); bm = C.c_double()
    lib().or_codon_qmat6(_p(_f(rel6), C.c_double), float(omega), _p(_f(pi), C.c_double), _p(Q, C.c_double), C.byref(bm))
    return Q, bm.value


def eigen(Q, pi):
    Q = _f(Q); n = Q.shape[0]
    ev = np.zeros(n); U = np.zeros((n, n)); Ui = np.zeros((n, n))
    lib().or_eigen(n, _p(Q, C.c_double), _p(_f(pi), C.c_double), _p(ev, C.c_double), _p(U, C.c_double), _p(Ui, C.c_double))
    return ev, U, Ui


def discrete_gamma(alpha, ncat):
    r = np.zeros(ncat)
    lib().or_discrete_gamma(float(alpha), int(ncat), _p(r, C.c_double))
    return r


def pmats(S, R, eval_scaled, U, Uinv, rates, pinv, has_pinv, t):
    n = R * S * S
    P, D1, D2 = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().or_pmats(S, R, _p(_f(eval_scaled), C.c_double), _p(_f(U), C.c_double), _p(_f(Uinv), C.c_double),
                   _p(_f(rates), C.c_double), float(pinv), int(has_pinv), float(t),
                   _p(P, C.c_double), _p(D1, C.c_double), _p(D2, C.c_double))
    return P.reshape(R, S, S), D1.reshape(R, S, S), D2.reshape(R, S, S)


def rescale_tables():
    incr = np.zeros(90, dtype=np.int32); th = np.zeros(90); mu = np.zeros(90)
    lib().or_rescale_tables(_p(incr, C.c_int), _p(th, C.c_double), _p(mu, C.c_double))
    return incr, th, mu


def set_threads(n: int, fast: bool = False):
    lib(fast).or_set_threads(int(n))


class OracleTree:
    """GARLI's CPU tree likelihood path (restated) on one alignment and topology."""

    def __init__(self, pd, child3, dlen, model, fast: bool = False):
        self.L = lib(fast)
        self.pd = pd
        self.child3 = np.ascontiguousarray(child3, dtype=np.int32)
        tips = np.ascontiguousarray(pd.tips, dtype=np.uint8)
        counts = np.ascontiguousarray(pd.counts, dtype=np.int32)
        cs = np.ascontiguousarray(pd.const_states, dtype=np.int32)
        self.t = self.L.or_tree_new(pd.ntax, pd.nstates, model.ncat, pd.npat, _p(self.child3, C.c_int),
                                    _p(_f(dlen), C.c_double), _p(tips, C.c_ubyte), _p(counts, C.c_int),
                                    int(pd.last_const), _p(cs, C.c_int))
        self.S, self.R, self.npat = pd.nstates, model.ncat, pd.npat
        self.set_model(model)

    def set_model(self, m):
        self.L.or_tree_set_model(self.t, _p(_f(m.eval_scaled), C.c_double), _p(_f(m.U), C.c_double),
                                 _p(_f(m.Uinv), C.c_double), _p(_f(m.pi), C.c_double),
                                 _p(_f(m.rates), C.c_double), _p(_f(m.probs), C.c_double), float(m.pinv),
                                 int(m.has_pinv))

    def close(self):
        if self.t:
            self.L.or_tree_free(self.t)
            self.t = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def score(self, root=0) -> float:
        return self.L.or_tree_score(self.t, root)

    def derivatives(self, node):
        out = np.zeros(3)
        rc = self.L.or_tree_derivs(self.t, node, _p(out, C.c_double))
        if rc:
            raise RuntimeError("oracle derivative failed")
        return out

    def optimize_branch(self, node, precision=0.01):
        return self.L.or_tree_nr_optimize(self.t, float(precision), node)

    def optimize_all_branches(self, precision=0.01):
        imp = self.L.or_tree_optimize_all(self.t, float(precision))
        return imp, self.L.or_tree_lnl(self.t)

    def set_branch_length(self, node, v):
        self.L.or_tree_set_blen(self.t, node, float(v))

    def branch_lengths(self):
        return np.array([self.L.or_tree_get_blen(self.t, i) for i in range(self.child3.shape[0])])

    def make_all_dirty(self):
        self.L.or_tree_dirty_all(self.t)

    @property
    def rescale_every(self):
        return self.L.or_tree_get_rescale_every(self.t)

    @rescale_every.setter
    def rescale_every(self, v):
        self.L.or_tree_set_rescale_every(self.t, int(v))

    def cla(self, node, which):
        arr = np.zeros((self.npat, self.R, self.S)); mult = np.zeros(self.npat, dtype=np.int32)
        rc = self.L.or_tree_get_cla(self.t, node, which, _p(arr, C.c_double), _p(mult, C.c_int))
        return (arr, mult) if rc == 0 else (None, None)

    def cla_rank(self, node, which):
        return self.L.or_tree_cla_rank(self.t, node, which)

    def cla_dirty(self, node, which):
        return bool(self.L.or_tree_cla_dirty(self.t, node, which))

    def site_lnl(self):
        out = np.zeros(self.npat)
        self.L.or_tree_site_lnl(self.t, _p(out, C.c_double))
        return out

    def counts(self):
        return {"cla": int(self.L.or_tree_cla_count(self.t)), "derivs": int(self.L.or_tree_deriv_count(self.t))}
