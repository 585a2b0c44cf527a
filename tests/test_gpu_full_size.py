"""Parity with the CPU oracle at the benchmark workloads' full sizes (needs a B200).

  dna_128x100k   DNA GTR+I+G4, 128 taxa x 100,000 sites (67,010 patterns)
  aa_64x20k      amino acids, 20 states +G4, 64 taxa x 20,000 sites
  codon_32x5k    codons, GY94 61 states, 32 taxa x 5,000 codons
  generation     GA generation: candidates of a 64-taxon tree, GTR+G4, 50,000 sites

For lnL the oracle builds its model with its own Q, discrete-gamma and eigen
code from the same parameters, so the whole chain (model math included) is
compared.  Derivatives and rescale counts are compared with both sides on the
engine's eigensystem: d1 near an optimum is a small sum of large terms of both
signs, and two eigensolvers' ulp-level differences in P(t) move it by more
than the arithmetic under test does.

Tolerances (no dependence on the pattern count):
  * plain FP64 form: lnL, d1 and d2 to 1e-8 relative (d1, d2 relative to
    max(1, |d|)); integer rescale counts exactly;
  * precision form (FP32 CLAs, power-of-two scalers), CUDA cores or tensor
    cores: |dlnL| <= 1e-4 absolute per tree; d1 and d2 to 1e-4 relative to
    max(1, |d|); optimised branch lengths to 1e-3 relative.
"""
import os

import numpy as np
import pytest

from garli_b200 import engine, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

PLAIN_REL = 1e-8
MIXED_ABS = 1e-4
DERIV_REL = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _setup():
    if engine.lib().gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")
    orc.set_threads(os.cpu_count() or 1)


_CACHE = {}


def _workload(name):
    """Workload and the oracle's scores on it (computed once per module)."""
    if name in _CACHE:
        return _CACHE[name]
    w = {"dna_128x100k": synth.dna_large, "aa_64x20k": synth.aa, "codon_32x5k": synth.codon}[name]()
    ot = orc.OracleTree(w.data, w.child3, w.dlen, w.model_with(orc))
    lnl = ot.score(0)
    ot.close()
    ot = orc.OracleTree(w.data, w.child3, w.dlen, w.model)
    ot.score(0)
    nn = w.child3.shape[0]
    # a sample of branches: tips, internal branches near the root and deep ones
    nodes = sorted({1, 2, w.data.ntax, w.data.ntax + 1, w.data.ntax + 2, nn // 2, nn - 2, nn - 1})
    derivs = {nd: ot.derivatives(nd) for nd in nodes}
    ot.make_all_dirty()
    ot.score(0)
    clas = {}
    for nd in (0, w.data.ntax + 1, nn - 1):
        arr, mult = ot.cla(nd, 0)
        if arr is not None:
            clas[nd] = mult
    ot.close()
    _CACHE[name] = (w, lnl, derivs, clas)
    return _CACHE[name]


@pytest.mark.parametrize("name", ["dna_128x100k", "aa_64x20k", "codon_32x5k"])
def test_plain_fp64_matches_oracle_at_full_size(name):
    w, lo, derivs, clas = _workload(name)
    inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model)
    lg = tree.score(0)
    assert abs(lg - lo) <= PLAIN_REL * abs(lo), (lg, lo)
    for nd, mult in clas.items():
        b = tree.cla_buffer(nd, 0)
        assert np.array_equal(inst.scale_factors(b), mult), nd
    for nd, o in derivs.items():
        g = tree.derivatives(nd)
        assert abs(g[0] - o[0]) <= PLAIN_REL * abs(o[0]), (nd, g, o)
        assert abs(g[1] - o[1]) <= PLAIN_REL * max(1.0, abs(o[1])), (nd, g, o)
        assert abs(g[2] - o[2]) <= PLAIN_REL * max(1.0, abs(o[2])), (nd, g, o)
    tree.close()
    inst.close()


@pytest.mark.parametrize("name,tc", [("dna_128x100k", False), ("aa_64x20k", False), ("aa_64x20k", True),
                                     ("codon_32x5k", False), ("codon_32x5k", True)])
def test_precision_form_matches_oracle_at_full_size(name, tc):
    w, lo, derivs, _ = _workload(name)
    inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model, mixed=True)
    if w.data.nstates > 4:
        inst.set_tensor_cores(tc)
    lg = tree.score(0)
    assert abs(lg - lo) <= MIXED_ABS, (lg, lo, lg - lo)
    for nd, o in derivs.items():
        g = tree.derivatives(nd)
        assert abs(g[0] - o[0]) <= MIXED_ABS, (nd, g, o)
        assert abs(g[1] - o[1]) <= DERIV_REL * max(1.0, abs(o[1])), (nd, g, o)
        assert abs(g[2] - o[2]) <= DERIV_REL * max(1.0, abs(o[2])), (nd, g, o)
    tree.close()
    inst.close()


def test_generation_candidates_match_oracle_at_full_size():
    """64 of the benchmark generation's candidates (64 taxa x 50,000 sites):
    batched precision form and GARLI's per-tree path against the oracle run on
    each candidate tree."""
    w, c3s, dls, conn = synth.batch_workload(seed=4)
    n = 64
    c3s, dls, conn = c3s[:n], dls[:n], conn[:n]
    m = w.model_with(orc)
    ref = []
    for i in range(n):
        ot = orc.OracleTree(w.data, c3s[i], dls[i], m)
        l0 = ot.score(0)
        X = int(conn[i])
        order = [int(c3s[i][X][0]), X, int(c3s[i][X][2])]
        for nd in order:
            ot.optimize_branch(nd, 0.01)
        lens = ot.branch_lengths()[order]
        ot.make_all_dirty()
        ref.append((l0, ot.score(0), lens))
        ot.close()
    for mixed, sequential in ((True, False), (False, True)):
        inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, n, mixed=mixed)
        out, lens = pop.score(c3s, dls, conn, 0.01, sequential=sequential)
        pop.close()
        inst.close()
        for i, (l0, lf, rl) in enumerate(ref):
            if mixed:
                assert abs(out[i, 0] - l0) <= MIXED_ABS, (i, out[i, 0], l0)
                assert abs(out[i, 1] - lf) <= MIXED_ABS, (i, out[i, 1], lf)
                assert np.allclose(lens[i], rl, rtol=1e-3, atol=1e-8), (i, lens[i], rl)
            else:
                assert abs(out[i, 0] - l0) <= PLAIN_REL * abs(l0), (i, out[i, 0], l0)
                assert abs(out[i, 1] - lf) <= PLAIN_REL * abs(lf), (i, out[i, 1], lf)
                assert np.allclose(lens[i], rl, rtol=1e-6, atol=1e-10), (i, lens[i], rl)
