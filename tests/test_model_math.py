"""The engine's host model math (gbm_*, model.cpp restated) against the oracle (no GPU)."""
import numpy as np
import pytest

from garli_b200 import engine, synth
from oracle import oracle as orc


def test_gtr_qmat_identical():
    rng = np.random.default_rng(5)
    for _ in range(5):
        pi = rng.dirichlet([10] * 4)
        rel = rng.gamma(2, 1, 6); rel /= rel[5]
        Qe, be = engine.gtr_qmat(rel, pi)
        Qo, bo = orc.gtr_qmat(rel, pi)
        assert np.array_equal(Qe, Qo) and be == bo


def test_aa_and_codon_qmat_identical():
    rng = np.random.default_rng(6)
    ex = rng.gamma(1, 1, 190); pi = rng.dirichlet([5] * 20)
    Qe, be = engine.aa_qmat(ex, pi); Qo, bo = orc.aa_qmat(ex, pi)
    assert np.allclose(Qe, Qo, rtol=1e-15, atol=0) and abs(be - bo) < 1e-15 * be
    f = rng.dirichlet([1] * 61)
    Qe, be = engine.codon_qmat(2.5, 0.3, f); Qo, bo = orc.codon_qmat(2.5, 0.3, f)
    assert np.allclose(Qe, Qo, rtol=1e-15, atol=0) and abs(be - bo) < 1e-14 * be
    assert np.allclose(Qe.sum(1), 0, atol=1e-14)
    r6 = rng.gamma(2, 1, 6)
    Qe, be = engine.codon_qmat6(r6, 0.4, f); Qo, bo = orc.codon_qmat6(r6, 0.4, f)
    assert np.allclose(Qe, Qo, rtol=1e-15, atol=0)


@pytest.mark.parametrize("n", [4, 20, 61])
def test_eigen_reconstructs_q(n):
    rng = np.random.default_rng(n)
    m = {4: synth.gtr_model, 20: synth.aa_model, 61: synth.codon_model}[n](rng)
    assert np.abs(m.U @ np.diag(m.eval) @ m.Uinv - m.Q).max() < 1e-13 * np.abs(m.Q).max()
    assert np.abs(m.U @ m.Uinv - np.eye(n)).max() < 1e-13


def test_discrete_gamma_engine_vs_oracle():
    for a, n in [(0.5, 4), (0.8, 4), (1.25046, 4), (1.34382, 5), (0.1, 4), (5.0, 6)]:
        e = engine.discrete_gamma(a, n)
        o = orc.discrete_gamma(a, n)
        assert np.allclose(e, o, rtol=1e-9, atol=1e-12), (a, n, e, o)
        assert abs(e.mean() - 1.0) < 1e-12


def test_host_pmats_match_oracle():
    rng = np.random.default_rng(3)
    m = synth.gtr_model(rng, pinv=0.2)
    P, _, _ = orc.pmats(4, 4, m.eval_scaled, m.U, m.Uinv, m.rates, m.pinv, m.has_pinv, 0.07)
    assert np.abs(m.pmats(0.07) - P).max() < 1e-15
