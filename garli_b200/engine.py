"""ctypes binding of the engine's C ABI (include/garli_b200.h).

This is the host-side mirror of the reference interface for the likelihood
path: ``Instance`` wraps the beagle-equivalent calls GARLI's
SubsetCalculationManager issues (subsetcalculationmanager.cpp), ``Tree`` wraps
the tree-level driver (Tree::Score, CalcDerivativesRateHet,
NewtonRaphsonOptimizeBranchLength, OptimizeAllBranches), and the ``*_qmat``,
``eigen`` and ``discrete_gamma`` helpers wrap the host model math
(model.cpp).  There is no fallback: if the shared library cannot be loaded
the import of the compute entry points raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

GB_SUCCESS = 0
GB_ERROR_UNINITIALIZED_INSTANCE = -4
GB_ERROR_OUT_OF_RANGE = -5
GB_ERROR_RESCALE_RETRY = -9
GB_FLAG_PLAIN_FP64 = 1 << 0
GB_FLAG_MIXED_FP32 = 1 << 1

_ERRORS = {
    -1: "GB_ERROR_GENERAL", -2: "GB_ERROR_OUT_OF_MEMORY", -3: "GB_ERROR_UNIDENTIFIED_EXCEPTION",
    -4: "GB_ERROR_UNINITIALIZED_INSTANCE", -5: "GB_ERROR_OUT_OF_RANGE", -6: "GB_ERROR_NO_RESOURCE",
    -7: "GB_ERROR_NO_IMPLEMENTATION", -8: "GB_ERROR_FLOATING_POINT", -9: "GB_ERROR_RESCALE_RETRY",
    -10: "GB_ERROR_NO_DEVICE",
}


class EngineError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = _lib_last_error()
        super().__init__(f"{where} failed: {_ERRORS.get(code, code)} {msg}")
        self.code = code


class ClaOperation(C.Structure):
    _fields_ = [("destClaIndex", C.c_int), ("childClaIndex1", C.c_int), ("childClaIndex2", C.c_int),
                ("transMatIndex1", C.c_int), ("transMatIndex2", C.c_int), ("opDepLevel", C.c_int)]


class TransMatOperation(C.Structure):
    _fields_ = [("destTransMatIndex", C.c_int), ("edgeLength", C.c_double), ("eigenIndex", C.c_int),
                ("calcDerivs", C.c_int)]


class ScoringOperation(C.Structure):
    _fields_ = [("destClaIndex", C.c_int), ("childClaIndex1", C.c_int), ("childClaIndex2", C.c_int),
                ("transMatIndex", C.c_int), ("derivatives", C.c_int)]


class ModelParams(C.Structure):
    """gb_model_params: GARLI's Model parameters of one tree (model.h)."""
    _fields_ = [("kind", C.c_int), ("stateCount", C.c_int), ("categoryCount", C.c_int), ("nst", C.c_int),
                ("hasPinv", C.c_int), ("alpha", C.c_double), ("pinv", C.c_double), ("maxPinv", C.c_double),
                ("omega", C.c_double), ("rel", C.c_double * 6), ("pi", C.c_double * 64)]


class InstanceDetails(C.Structure):
    _fields_ = [("resourceNumber", C.c_int), ("flags", C.c_long), ("paddedPatterns", C.c_int),
                ("deviceBytes", C.c_longlong), ("deviceName", C.c_char * 64)]


_LIB = None

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_U8 = C.POINTER(C.c_ubyte)
_LL = C.POINTER(C.c_longlong)

# name -> (restype, argtypes); every symbol declared in include/garli_b200.h
SIGNATURES = {
    "gb_get_device_count": (C.c_int, []),
    "gb_create_instance": (C.c_int, [C.c_int] * 8 + [C.c_long, C.POINTER(InstanceDetails)]),
    "gb_finalize_instance": (C.c_int, [C.c_int]),
    "gb_set_tip_states": (C.c_int, [C.c_int, C.c_int, _U8]),
    "gb_set_pattern_weights": (C.c_int, [C.c_int, _I]),
    "gb_set_constant_patterns": (C.c_int, [C.c_int, C.c_int, _I]),
    "gb_set_state_frequencies": (C.c_int, [C.c_int, _D]),
    "gb_set_category_rates": (C.c_int, [C.c_int, _D]),
    "gb_set_category_weights": (C.c_int, [C.c_int, _D]),
    "gb_set_invariant_sites": (C.c_int, [C.c_int, C.c_double, C.c_int]),
    "gb_set_eigen_decomposition": (C.c_int, [C.c_int, C.c_int, _D, _D, _D]),
    "gb_update_transition_matrices": (C.c_int, [C.c_int, C.POINTER(TransMatOperation), C.c_int]),
    "gb_set_transition_matrix": (C.c_int, [C.c_int, C.c_int, _D, _D, _D]),
    "gb_update_partials": (C.c_int, [C.c_int, C.POINTER(ClaOperation), C.c_int, C.c_int]),
    "gb_calculate_edge": (C.c_int, [C.c_int, C.POINTER(ScoringOperation), _D]),
    "gb_get_site_log_likelihoods": (C.c_int, [C.c_int, _D]),
    "gb_get_site_derivatives": (C.c_int, [C.c_int, _D, _D]),
    "gb_get_partials": (C.c_int, [C.c_int, C.c_int, _D]),
    "gb_get_scale_factors": (C.c_int, [C.c_int, C.c_int, _I]),
    "gb_get_transition_matrix": (C.c_int, [C.c_int, C.c_int, C.c_int, _D]),
    "gb_get_rescale_rank": (C.c_int, [C.c_int, C.c_int]),
    "gb_get_partials_pool": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), _LL]),
    "gb_get_instance_shape": (C.c_int, [C.c_int, _I]),
    "gb_get_launch_count": (C.c_longlong, [C.c_int]),
    "gb_synchronize": (C.c_int, [C.c_int]),
    "gb_last_error": (C.c_char_p, []),
    "gb_get_stream": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "gb_set_kernel_timing": (C.c_int, [C.c_int, C.c_int]),
    "gb_get_kernel_timing": (C.c_int, [C.c_int, _D]),
    "gb_set_branch_lengths": (C.c_int, [C.c_int, _D, C.c_int]),
    "gb_get_branch_lengths": (C.c_int, [C.c_int, _D, C.c_int]),
    "gb_newton_pass": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _D]),
    "gb_get_newton_state": (C.c_int, [C.c_int, C.c_int, _D]),
    "gb_set_pass_mode": (C.c_int, [C.c_int, C.c_int]),
    "gb_set_pass_trace": (C.c_int, [C.c_int, C.c_int]),
    "gb_get_pass_trace": (C.c_int, [C.c_int, C.POINTER(C.c_ulonglong), C.c_int]),
    "gbt_set_device_newton": (C.c_int, [C.c_int, C.c_int]),
    "gb_batch_newton": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                  C.c_int, C.c_double, C.c_double, C.c_double, _D]),
    "gb_set_batch_tuning": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "gb_get_batch_tuning": (C.c_int, [C.c_int, _I]),
    "gb_get_batch_timing": (C.c_int, [C.c_int, _D]),
    "gb_set_tensor_cores": (C.c_int, [C.c_int, C.c_int]),
    "gb_set_cla_tuning": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "gb_get_cla_tuning": (C.c_int, [C.c_int, _I]),
    "gb_set_buffer_precision": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "gb_set_eigen_from_rate_matrices": (C.c_int, [C.c_int, C.c_int, _I, _D, _D, _D, _I]),
    "gbp_create": (C.c_int, [C.c_int, C.c_int, _I, _D, C.c_int]),
    "gbp_destroy": (C.c_int, [C.c_int]),
    "gbp_invalidate": (C.c_int, [C.c_int]),
    "gbp_score_candidates": (C.c_int, [C.c_int, C.c_int, _I, _D, _I, C.c_double, C.c_int, _D, _D]),
    "gbp_get_counters": (C.c_int, [C.c_int, _LL]),
    "gbp_get_byte_counters": (C.c_int, [C.c_int, _D]),
    "gb_set_batch_phase_timing": (C.c_int, [C.c_int, C.c_int]),
    "gb_get_batch_phase_timing": (C.c_int, [C.c_int, _D]),
    "gb_edge_loglik_static": (C.c_int, [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 10 + [C.c_double, C.c_int, C.c_int,
                                                                                          C.c_void_p, C.c_void_p]),
    "gbm_gtr_qmat": (C.c_int, [_D, _D, _D, _D]),
    "gbm_aa_qmat": (C.c_int, [_D, _D, _D, _D]),
    "gbm_codon_qmat": (C.c_int, [C.c_double, C.c_double, _D, _D, _D]),
    "gbm_codon_qmat6": (C.c_int, [_D, C.c_double, _D, _D, _D]),
    "gbm_eigen": (C.c_int, [C.c_int, _D, _D, _D, _D, _D]),
    "gbm_discrete_gamma": (C.c_int, [C.c_double, C.c_int, _D]),
    "gbt_create": (C.c_int, [C.c_int, C.c_int, _I, _D]),
    "gbt_destroy": (C.c_int, [C.c_int]),
    "gbt_set_model": (C.c_int, [C.c_int, _D, _D, _D, C.c_double, _D, _D, _D, C.c_double, C.c_int]),
    "gbt_score": (C.c_int, [C.c_int, C.c_int, _D]),
    "gbt_derivatives": (C.c_int, [C.c_int, C.c_int, _D]),
    "gbt_set_branch_length": (C.c_int, [C.c_int, C.c_int, C.c_double]),
    "gbt_get_branch_lengths": (C.c_int, [C.c_int, _D]),
    "gbt_make_all_dirty": (C.c_int, [C.c_int]),
    "gbt_optimize_branch": (C.c_int, [C.c_int, C.c_double, C.c_int, _D]),
    "gbt_optimize_all_branches": (C.c_int, [C.c_int, C.c_double, _D]),
    "gbt_get_rescale_every": (C.c_int, [C.c_int]),
    "gbt_set_rescale_every": (C.c_int, [C.c_int, C.c_int]),
    "gbt_get_counters": (C.c_int, [C.c_int, _LL]),
    "gbt_cla_buffer": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "gbt_score_models": (C.c_int, [C.c_int, C.c_int, _I, _D]),
    "gbt_get_instance": (C.c_int, [C.c_int]),
    "gb_set_model_slot": (C.c_int, [C.c_int, C.c_int, _D, _D, _D, C.c_double, C.c_int]),
    "gb_calculate_edges": (C.c_int, [C.c_int, C.POINTER(ScoringOperation), _I, C.c_int, _D]),
    "gb_get_instance_capacity": (C.c_int, [C.c_int, _I]),
    "gbo_create": (C.c_int, [C.c_int, C.POINTER(ModelParams), _D]),
    "gbo_destroy": (C.c_int, [C.c_int]),
    "gbo_get_model": (C.c_int, [C.c_int, C.POINTER(ModelParams)]),
    "gbo_set_model": (C.c_int, [C.c_int, C.POINTER(ModelParams)]),
    "gbo_optimize_parameter": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                         _D]),
    "gbo_optimize_model": (C.c_int, [C.c_int, C.c_int, C.c_double, _D]),
    "gbo_final_optimization": (C.c_int, [C.c_int, C.c_double, C.c_int, C.c_int, _D]),
    "gbo_set_batching": (C.c_int, [C.c_int, C.c_int]),
    "gbo_get_counters": (C.c_int, [C.c_int, _LL]),
    "gbo_get_trace": (C.c_int, [C.c_int, _D, _D, C.c_int, _D]),
}


def lib_path() -> str:
    return _build.LIB


def lib() -> C.CDLL:
    """Load (building first if the .so is absent or stale) the engine library."""
    global _LIB
    if _LIB is None:
        path = _build.build() if _build.nvcc_available() else _build.LIB
        if not os.path.exists(path):
            raise RuntimeError(f"garli_b200 engine library missing: {path} (run python -m garli_b200.build)")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _lib_last_error() -> str:
    try:
        return (lib().gb_last_error() or b"").decode()
    except Exception:  # pragma: no cover
        return ""


def _p(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def _chk(rc: int, where: str) -> int:
    if rc < 0:
        raise EngineError(rc, where)
    return rc


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


# ---------------------------------------------------------------- model math
def gtr_qmat(rel6, pi4):
    Q = np.zeros((4, 4)); bm = C.c_double()
    _chk(lib().gbm_gtr_qmat(_p(_f64(rel6), C.c_double), _p(_f64(pi4), C.c_double), _p(Q, C.c_double), C.byref(bm)), "gbm_gtr_qmat")
    return Q, bm.value


def aa_qmat(exch190, pi20):
    Q = np.zeros((20, 20)); bm = C.c_double()
    _chk(lib().gbm_aa_qmat(_p(_f64(exch190), C.c_double), _p(_f64(pi20), C.c_double), _p(Q, C.c_double), C.byref(bm)), "gbm_aa_qmat")
    return Q, bm.value


def codon_qmat(kappa, omega, pi61):
    Q = np.zeros((61, 61)); bm = C.c_double()
    _chk(lib().gbm_codon_qmat(kappa, omega, _p(_f64(pi61), C.c_double), _p(Q, C.c_double), C.byref(bm)), "gbm_codon_qmat")
    return Q, bm.value


def codon_qmat6(rel6, omega, pi61):
    Q = np.zeros((61, 61)); bm = C.c_double()
    _chk(lib().gbm_codon_qmat6(_p(_f64(rel6), C.c_double), float(omega), _p(_f64(pi61), C.c_double), _p(Q, C.c_double), C.byref(bm)), "gbm_codon_qmat6")
    return Q, bm.value


def eigen(Q, pi):
    Q = _f64(Q); pi = _f64(pi); n = Q.shape[0]
    ev = np.zeros(n); U = np.zeros((n, n)); Ui = np.zeros((n, n))
    _chk(lib().gbm_eigen(n, _p(Q, C.c_double), _p(pi, C.c_double), _p(ev, C.c_double), _p(U, C.c_double), _p(Ui, C.c_double)), "gbm_eigen")
    return ev, U, Ui


def discrete_gamma(alpha: float, ncat: int) -> np.ndarray:
    r = np.zeros(ncat)
    _chk(lib().gbm_discrete_gamma(float(alpha), int(ncat), _p(r, C.c_double)), "gbm_discrete_gamma")
    return r


@dataclass
class Model:
    """A substitution model in GARLI's terms (Model class, model.h)."""

    nstates: int
    pi: np.ndarray
    Q: np.ndarray
    blen_mult: float
    eval: np.ndarray  # unscaled eigenvalues of Q
    U: np.ndarray
    Uinv: np.ndarray
    rates: np.ndarray  # rateMults
    probs: np.ndarray  # rateProbs = (1-pinv)/ncat
    pinv: float = 0.0
    has_pinv: bool = False

    @property
    def ncat(self) -> int:
        return len(self.rates)

    @property
    def eval_scaled(self) -> np.ndarray:
        return self.eval * self.blen_mult

    def pmats(self, t: float) -> np.ndarray:
        """P(t) for every category ([R, S, S]) with the engine's formula (host copy, for simulation)."""
        sev = self.eval_scaled[None, :] * self.rates[:, None]
        if self.has_pinv:
            sev = sev / (1.0 - self.pinv)
        e = np.exp(sev * t)
        P = np.einsum("ik,rk,kj->rij", self.U, e, self.Uinv)
        return np.maximum(P, 0.0)


def make_model(nstates, Q, blen_mult, pi, rates, pinv=0.0, has_pinv=False) -> Model:
    ev, U, Ui = eigen(Q, pi)
    rates = _f64(rates)
    probs = np.full(len(rates), (1.0 - pinv) / len(rates))
    return Model(nstates, _f64(pi), _f64(Q), blen_mult, ev, U, Ui, rates, probs, float(pinv), bool(has_pinv))


# ---------------------------------------------------------------- instance
class Instance:
    """One engine instance (a beagle instance in GARLI's BEAGLE build)."""

    def __init__(self, ntip, nbuf, nstates, npat, ncat, nmat, neigen=1, device=0, mixed=False):
        self.details = InstanceDetails()
        flags = GB_FLAG_MIXED_FP32 if mixed else GB_FLAG_PLAIN_FP64
        h = lib().gb_create_instance(ntip, nbuf, nstates, npat, neigen, nmat, ncat, device, flags, C.byref(self.details))
        _chk(h, "gb_create_instance")
        self.h = h
        self.ntip, self.nbuf, self.S, self.npat, self.R, self.nmat = ntip, nbuf, nstates, npat, ncat, nmat
        self.mixed = mixed

    def close(self):
        if getattr(self, "h", -1) >= 0:
            lib().gb_finalize_instance(self.h)
            self.h = -1

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_data(self, pd):
        for t in range(pd.ntax):
            row = np.ascontiguousarray(pd.tips[t], dtype=np.uint8)
            _chk(lib().gb_set_tip_states(self.h, t, _p(row, C.c_ubyte)), "gb_set_tip_states")
        _chk(lib().gb_set_pattern_weights(self.h, _p(_i32(pd.counts), C.c_int)), "gb_set_pattern_weights")
        _chk(lib().gb_set_constant_patterns(self.h, pd.last_const, _p(_i32(pd.const_states), C.c_int)), "gb_set_constant_patterns")

    def set_model(self, m: Model, eigen_index=0):
        L = lib()
        _chk(L.gb_set_eigen_decomposition(self.h, eigen_index, _p(_f64(m.U), C.c_double), _p(_f64(m.Uinv), C.c_double), _p(_f64(m.eval_scaled), C.c_double)), "gb_set_eigen_decomposition")
        _chk(L.gb_set_state_frequencies(self.h, _p(_f64(m.pi), C.c_double)), "gb_set_state_frequencies")
        _chk(L.gb_set_category_rates(self.h, _p(_f64(m.rates), C.c_double)), "gb_set_category_rates")
        _chk(L.gb_set_category_weights(self.h, _p(_f64(m.probs), C.c_double)), "gb_set_category_weights")
        _chk(L.gb_set_invariant_sites(self.h, float(m.pinv), int(m.has_pinv)), "gb_set_invariant_sites")

    def update_transition_matrices(self, ops):
        arr = (TransMatOperation * len(ops))(*[TransMatOperation(int(a), float(b), int(c), int(d)) for a, b, c, d in ops])
        _chk(lib().gb_update_transition_matrices(self.h, arr, len(ops)), "gb_update_transition_matrices")

    def update_partials(self, ops, rescale_every=16):
        arr = (ClaOperation * len(ops))(*[ClaOperation(*[int(x) for x in o]) for o in ops])
        return _chk(lib().gb_update_partials(self.h, arr, len(ops), rescale_every), "gb_update_partials")

    def calculate_edge(self, partial, child, mat, derivatives=False, check=True):
        op = ScoringOperation(-1, partial, child, mat, int(derivatives))
        out = np.zeros(3)
        rc = lib().gb_calculate_edge(self.h, C.byref(op), _p(out, C.c_double))
        if check:
            _chk(rc, "gb_calculate_edge")
        return (out, rc) if not check else out

    def site_lnl(self):
        out = np.zeros(self.npat)
        _chk(lib().gb_get_site_log_likelihoods(self.h, _p(out, C.c_double)), "gb_get_site_log_likelihoods")
        return out

    def site_derivatives(self):
        """Per-pattern d1, d2 of the last derivative edge evaluation."""
        a, b = np.zeros(self.npat), np.zeros(self.npat)
        _chk(lib().gb_get_site_derivatives(self.h, _p(a, C.c_double), _p(b, C.c_double)), "gb_get_site_derivatives")
        return a, b

    def partials(self, buf):
        out = np.zeros((self.npat, self.R, self.S))
        _chk(lib().gb_get_partials(self.h, buf, _p(out, C.c_double)), "gb_get_partials")
        return out

    def scale_factors(self, buf):
        out = np.zeros(self.npat, dtype=np.int32)
        _chk(lib().gb_get_scale_factors(self.h, buf, _p(out, C.c_int)), "gb_get_scale_factors")
        return out

    def transition_matrix(self, mat, which=0):
        out = np.zeros((self.R, self.S, self.S))
        _chk(lib().gb_get_transition_matrix(self.h, mat, which, _p(out, C.c_double)), "gb_get_transition_matrix")
        return out

    def launch_count(self) -> int:
        return int(lib().gb_get_launch_count(self.h))

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        _chk(lib().gb_get_stream(self.h, C.byref(p)), "gb_get_stream")
        return p.value or 0

    def set_kernel_timing(self, on: bool):
        _chk(lib().gb_set_kernel_timing(self.h, int(on)), "gb_set_kernel_timing")

    def kernel_timing(self) -> dict:
        out = np.zeros(7)
        _chk(lib().gb_get_kernel_timing(self.h, _p(out, C.c_double)), "gb_get_kernel_timing")
        return {"cla_ms": out[0], "cla_launches": int(out[1]), "pattern_updates": int(out[2]),
                "edge_ms": out[3], "edge_evals": int(out[4]), "cla_bytes": out[5], "cla_fp64_instr": out[6]}

    def synchronize(self):
        _chk(lib().gb_synchronize(self.h), "gb_synchronize")

    def set_eigen_from_q(self, eigen_indices, Qs, pis, blen_mults):
        """Eigensystems of rate matrices computed on the device (one CTA per model);
        returns the Jacobi sweeps each took."""
        idx = _i32(eigen_indices)
        n = len(idx)
        sw = np.zeros(n, dtype=np.int32)
        _chk(lib().gb_set_eigen_from_rate_matrices(self.h, n, _p(idx, C.c_int), _p(_f64(Qs), C.c_double),
                                                   _p(_f64(pis), C.c_double), _p(_f64(blen_mults), C.c_double),
                                                   _p(sw, C.c_int)), "gb_set_eigen_from_rate_matrices")
        return sw

    def set_tensor_cores(self, on: bool):
        _chk(lib().gb_set_tensor_cores(self.h, int(on)), "gb_set_tensor_cores")

    def set_cla_tuning(self, level_blocks_per_sm=-1, nstate_tile=-1):
        _chk(lib().gb_set_cla_tuning(self.h, int(level_blocks_per_sm), int(nstate_tile)), "gb_set_cla_tuning")

    def cla_tuning(self) -> dict:
        out = np.zeros(3, dtype=np.int32)
        _chk(lib().gb_get_cla_tuning(self.h, _p(out, C.c_int)), "gb_get_cla_tuning")
        return {"level_blocks_per_sm": int(out[0]), "nstate_tile": int(out[1]), "pending": bool(out[2])}

    def set_model_slot(self, slot, pi, rates, weights, pinv=0.0, has_pinv=False):
        """Frequencies, category rates / weights and pinv read with eigen index ``slot``."""
        _chk(lib().gb_set_model_slot(self.h, int(slot), _p(_f64(pi), C.c_double), _p(_f64(rates), C.c_double),
                                     _p(_f64(weights), C.c_double), float(pinv), int(has_pinv)),
             "gb_set_model_slot")

    def capacity(self) -> tuple:
        out = np.zeros(3, dtype=np.int32)
        _chk(lib().gb_get_instance_capacity(self.h, _p(out, C.c_int)), "gb_get_instance_capacity")
        return int(out[0]), int(out[1]), int(out[2])

    def set_pass_mode(self, persistent: bool):
        _chk(lib().gb_set_pass_mode(self.h, int(persistent)), "gb_set_pass_mode")


class Tree:
    """GARLI's tree-level entry points on one instance (gbt_* in the ABI)."""

    def __init__(self, inst: Instance, child3: np.ndarray, dlen: np.ndarray):
        self.inst = inst
        self.child3 = _i32(child3)
        self.ntax = (self.child3.shape[0] + 2) // 2
        h = lib().gbt_create(inst.h, self.ntax, _p(self.child3, C.c_int), _p(_f64(dlen), C.c_double))
        _chk(h, "gbt_create")
        self.h = h

    def close(self):
        if getattr(self, "h", -1) >= 0:
            lib().gbt_destroy(self.h)
            self.h = -1

    def set_model(self, m: Model):
        _chk(lib().gbt_set_model(self.h, _p(_f64(m.eval), C.c_double), _p(_f64(m.U), C.c_double), _p(_f64(m.Uinv), C.c_double), float(m.blen_mult), _p(_f64(m.pi), C.c_double), _p(_f64(m.rates), C.c_double), _p(_f64(m.probs), C.c_double), float(m.pinv), int(m.has_pinv)), "gbt_set_model")

    def score(self, root=0) -> float:
        out = np.zeros(3)
        _chk(lib().gbt_score(self.h, root, _p(out, C.c_double)), "gbt_score")
        return float(out[0])

    def derivatives(self, node):
        out = np.zeros(3)
        _chk(lib().gbt_derivatives(self.h, node, _p(out, C.c_double)), "gbt_derivatives")
        return out

    def set_branch_length(self, node, v):
        _chk(lib().gbt_set_branch_length(self.h, node, float(v)), "gbt_set_branch_length")

    def branch_lengths(self):
        out = np.zeros(self.child3.shape[0])
        _chk(lib().gbt_get_branch_lengths(self.h, _p(out, C.c_double)), "gbt_get_branch_lengths")
        return out

    def make_all_dirty(self):
        _chk(lib().gbt_make_all_dirty(self.h), "gbt_make_all_dirty")

    def optimize_branch(self, node, precision=0.01) -> float:
        out = np.zeros(1)
        _chk(lib().gbt_optimize_branch(self.h, float(precision), node, _p(out, C.c_double)), "gbt_optimize_branch")
        return float(out[0])

    def optimize_all_branches(self, precision=0.01):
        out = np.zeros(2)
        _chk(lib().gbt_optimize_all_branches(self.h, float(precision), _p(out, C.c_double)), "gbt_optimize_all_branches")
        return float(out[0]), float(out[1])

    def set_device_newton(self, on: bool):
        _chk(lib().gbt_set_device_newton(self.h, int(on)), "gbt_set_device_newton")

    @property
    def rescale_every(self) -> int:
        return _chk(lib().gbt_get_rescale_every(self.h), "gbt_get_rescale_every")

    @rescale_every.setter
    def rescale_every(self, v: int):
        _chk(lib().gbt_set_rescale_every(self.h, int(v)), "gbt_set_rescale_every")

    def counters(self) -> dict:
        out = np.zeros(5, dtype=np.int64)
        _chk(lib().gbt_get_counters(self.h, _p(out, C.c_longlong)), "gbt_get_counters")
        return {"cla_ops": int(out[0]), "pattern_updates": int(out[1]), "edge_evals": int(out[2]),
                "scores": int(out[3]), "rescale_retries": int(out[4])}

    def cla_buffer(self, node, which) -> int:
        return lib().gbt_cla_buffer(self.h, node, which)


    def score_models(self, slots) -> np.ndarray:
        """Full rescores of the tree under the models in eigen / model slots ``slots``."""
        sl = _i32(slots)
        out = np.zeros(len(sl))
        _chk(lib().gbt_score_models(self.h, len(sl), _p(sl, C.c_int), _p(out, C.c_double)), "gbt_score_models")
        return out


# GB_MODEL_*, GB_PARAM_*, GB_OPT_* (include/garli_b200.h)
MODEL_NUCLEOTIDE, MODEL_AMINO_ACID, MODEL_CODON = 0, 1, 2
PARAM_ALPHA, PARAM_PINV, PARAM_STATE_FREQ, PARAM_REL_RATE, PARAM_OMEGA = 0, 1, 2, 3, 4
OPT_ALPHA, OPT_PINV, OPT_FREQS, OPT_RATES, OPT_OMEGA = 1, 2, 4, 8, 16


def model_params(kind, pi, rel=None, alpha=0.5, ncat=1, pinv=None, max_pinv=0.0, omega=1.0, nst=6) -> ModelParams:
    """gb_model_params from plain values (pinv None: no invariant-sites class)."""
    m = ModelParams()
    m.kind = kind
    m.stateCount = len(pi)
    m.categoryCount = ncat
    m.nst = nst
    m.hasPinv = 0 if pinv is None else 1
    m.alpha = alpha
    m.pinv = 0.0 if pinv is None else float(pinv)
    m.maxPinv = max_pinv
    m.omega = omega
    for i, v in enumerate(rel if rel is not None else [1.0] * 6):
        m.rel[i] = float(v)
    for i, v in enumerate(pi):
        m.pi[i] = float(v)
    return m


class ModelOptimizer:
    """GARLI's model-parameter optimisation of one tree (gbo_* in the ABI)."""

    def __init__(self, tree: "Tree", params: ModelParams, exch=None):
        self.tree = tree
        ex = None if exch is None else _f64(exch)
        h = lib().gbo_create(tree.h, C.byref(params), None if ex is None else _p(ex, C.c_double))
        _chk(h, "gbo_create")
        self.h = h

    def close(self):
        if getattr(self, "h", -1) >= 0:
            lib().gbo_destroy(self.h)
            self.h = -1

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> ModelParams:
        m = ModelParams()
        _chk(lib().gbo_get_model(self.h, C.byref(m)), "gbo_get_model")
        return m

    def set_params(self, m: ModelParams):
        _chk(lib().gbo_set_model(self.h, C.byref(m)), "gbo_set_model")

    def optimize_parameter(self, param, which, precision, low, high, target_digits=9.0):
        """OptimizeBoundedParameter: (improvement, final lnL)."""
        out = np.zeros(2)
        _chk(lib().gbo_optimize_parameter(self.h, param, which, float(precision), float(low), float(high),
                                          float(target_digits), _p(out, C.c_double)), "gbo_optimize_parameter")
        return float(out[0]), float(out[1])

    def optimize_model(self, mask, precision) -> np.ndarray:
        out = np.zeros(5)
        _chk(lib().gbo_optimize_model(self.h, int(mask), float(precision), _p(out, C.c_double)),
             "gbo_optimize_model")
        return out

    def final_optimization(self, branch_precision=0.01, mask=31, max_passes=0):
        """BetterFinalOptimization: (final lnL, passes, model evaluations)."""
        out = np.zeros(3)
        _chk(lib().gbo_final_optimization(self.h, float(branch_precision), int(mask), int(max_passes),
                                          _p(out, C.c_double)), "gbo_final_optimization")
        return float(out[0]), int(out[1]), int(out[2])

    def set_batching(self, depth: int):
        _chk(lib().gbo_set_batching(self.h, int(depth)), "gbo_set_batching")

    def trace(self):
        """(initial lnL, values, scores) of the last OptimizeBoundedParameter call."""
        ini = C.c_double()
        n = _chk(lib().gbo_get_trace(self.h, None, None, 0, C.byref(ini)), "gbo_get_trace")
        v, sc = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        _chk(lib().gbo_get_trace(self.h, _p(v, C.c_double), _p(sc, C.c_double), n, None), "gbo_get_trace")
        return ini.value, v[:n], sc[:n]

    def counters(self) -> dict:
        out = np.zeros(3, dtype=np.int64)
        _chk(lib().gbo_get_counters(self.h, _p(out, C.c_longlong)), "gbo_get_counters")
        return {"evaluations": int(out[0]), "models_scored": int(out[1]), "score_calls": int(out[2])}


def model_engine(pd, child3, dlen, params: ModelParams, kmax=8, exch=None, device=0):
    """Instance, Tree and ModelOptimizer for model-parameter optimisation of one
    tree: room for kmax candidate models per batched rescore."""
    ntax = pd.ntax
    nnodes = 2 * ntax - 2
    nint = ntax - 2
    inst = Instance(ntax, (3 + kmax) * nint, pd.nstates, pd.npat, params.categoryCount, (kmax + 1) * nnodes,
                    neigen=kmax + 1, device=device)
    inst.set_data(pd)
    tree = Tree(inst, child3, dlen)
    opt = ModelOptimizer(tree, params, exch)
    return inst, tree, opt


def tree_engine(pd, child3, dlen, model: Model, device=0, mixed=False):
    """Create an instance sized for one tree over ``pd`` and its Tree driver."""
    ntax = pd.ntax
    nnodes = 2 * ntax - 2
    inst = Instance(ntax, 3 * (ntax - 2), pd.nstates, pd.npat, model.ncat, nnodes, device=device, mixed=mixed)
    inst.set_data(pd)
    tree = Tree(inst, child3, dlen)
    tree.set_model(model)
    return inst, tree


# ---------------------------------------------------------------- GA population
class Population:
    """A GA generation's candidates scored on one instance (gbp_* ABI).

    ``base`` is the parent tree (child3, dlen); candidates are trees on the same
    node numbers with the connector node of their move (synth.ga_candidates)."""

    def __init__(self, inst: Instance, child3: np.ndarray, dlen: np.ndarray, nmat: int):
        self.inst = inst
        self.nnodes = child3.shape[0]
        c3 = _i32(np.asarray(child3).reshape(-1))
        h = lib().gbp_create(inst.h, (self.nnodes + 2) // 2, _p(c3, C.c_int), _p(_f64(dlen), C.c_double), nmat)
        _chk(h, "gbp_create")
        self.h = h

    def close(self):
        if getattr(self, "h", -1) >= 0:
            lib().gbp_destroy(self.h)
            self.h = -1

    def score(self, child3s, dlens, connectors, precision=0.01, sequential=False):
        """Per candidate: (rescore lnL, optimised lnL, improvement, evaluations) and
        the optimised lengths of connector.left, connector, connector.right."""
        n = len(connectors)
        c3 = _i32(np.asarray(child3s).reshape(-1))
        dl = _f64(np.asarray(dlens).reshape(-1))
        cn = _i32(connectors)
        out = np.zeros((n, 4))
        lens = np.zeros((n, 3))
        _chk(lib().gbp_score_candidates(self.h, n, _p(c3, C.c_int), _p(dl, C.c_double), _p(cn, C.c_int),
                                        float(precision), int(sequential), _p(out, C.c_double),
                                        _p(lens, C.c_double)), "gbp_score_candidates")
        return out, lens

    def counters(self) -> dict:
        out = np.zeros(6, dtype=np.int64)
        _chk(lib().gbp_get_counters(self.h, out.ctypes.data_as(_LL)), "gbp_get_counters")
        return {"cla_ops": int(out[0]), "pattern_updates": int(out[1]), "deriv_evals": int(out[2]),
                "base_cla_ops": int(out[3]), "edge_evals": int(out[4]), "alg_bytes": int(out[5])}

    def set_tuning(self, tiles_per_item: int, chunks_per_item: int):
        """Work-item sizes of the batched pass (0, 0: autotune on the next call)."""
        _chk(lib().gb_set_batch_tuning(self.inst.h, int(tiles_per_item), int(chunks_per_item)),
             "gb_set_batch_tuning")

    def byte_counters(self) -> dict:
        """Algorithmic bytes of the last call by phase."""
        out = np.zeros(3)
        _chk(lib().gbp_get_byte_counters(self.h, _p(out, C.c_double)), "gbp_get_byte_counters")
        return {"levels": float(out[0]), "coefficients": float(out[1]), "sweeps": float(out[2])}

    def set_phase_timing(self, on: bool):
        _chk(lib().gb_set_batch_phase_timing(self.inst.h, int(on)), "gb_set_batch_phase_timing")

    def phase_timing(self) -> dict:
        """Accumulated CUDA-event ms and launches per phase of the batched pass."""
        out = np.zeros(6)
        _chk(lib().gb_get_batch_phase_timing(self.inst.h, _p(out, C.c_double)), "gb_get_batch_phase_timing")
        return {k: {"ms": float(out[2 * i]), "launches": int(out[2 * i + 1])}
                for i, k in enumerate(("levels", "coefficients", "sweeps"))}

    def batch_timing(self) -> dict:
        out = np.zeros(2)
        _chk(lib().gb_get_batch_timing(self.inst.h, _p(out, C.c_double)), "gb_get_batch_timing")
        return {"ms": float(out[0]), "launches": int(out[1])}

    def tuning(self) -> dict:
        out = np.zeros(3, dtype=np.int32)
        _chk(lib().gb_get_batch_tuning(self.inst.h, _p(out, C.c_int)), "gb_get_batch_tuning")
        return {"tiles_per_item": int(out[0]), "chunks_per_item": int(out[1]), "cuda_graph": bool(out[2])}


def population_engine(pd, child3, dlen, model: Model, ncand: int, device=0, mixed=True, extra_bufs_per_cand=40):
    """Instance + Population sized for ``ncand`` candidates of a base tree."""
    ntax = pd.ntax
    nnodes = 2 * ntax - 2
    nbuf = 6 * (ntax - 2) + ncand * (extra_bufs_per_cand + 1)  # base CLAs may take two slots (FP64)
    nmat = nnodes + ncand * 8
    inst = Instance(ntax, nbuf, pd.nstates, pd.npat, model.ncat, nmat, device=device, mixed=mixed)
    inst.set_data(pd)
    inst.set_model(model)
    pop = Population(inst, child3, dlen, nmat)
    return inst, pop
