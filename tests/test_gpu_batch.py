"""Batched GA-population scoring (gb_batch_newton through the gbp_* layer) against
the CPU oracle and against GARLI's per-tree path on the same GPU.

Each candidate is the base tree after one SPR/NNI move; it is rescored and its
three branches at the connector nd are optimised in GARLI's order nd->left, nd,
nd->right (optimization.cpp:882-884).  The oracle does exactly that on the
candidate tree with GARLI's CPU code path.

Both GTR+G4 and GTR+I+G4 (the +I term enters every site likelihood of the
constant patterns, scaled by the pattern's scalers).

Tolerances:
  * plain FP64 per-tree path: rescore lnL to 1e-8 relative of the oracle;
    optimised lengths to 1e-6 relative, optimised lnL to 1e-8 relative;
  * plain FP64 batched vs plain per-tree: same plan, different summation
    partition: lnL to 1e-10 relative, lengths to 1e-8 relative;
  * precision form batched (FP32 CLAs): |dlnL| <= 1e-4
    absolute per tree, lengths to 1e-3 relative.
"""
import numpy as np
import pytest

from garli_b200 import engine, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["gtr_g4", "gtr_i_g4"])
def case(request):
    if engine.lib().gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")
    pinv = (0.05, 0.3) if request.param == "gtr_i_g4" else None
    w = synth.make_dna(24, 1500, seed=41, pinv_range=pinv)
    c3s, dls, conn = synth.ga_candidates(w.child3, w.dlen, 12, seed=42, radius_range=(1, 6))
    ref = []
    om = w.model_with(orc)
    for i in range(len(conn)):
        ot = orc.OracleTree(w.data, c3s[i], dls[i], om)
        l0 = ot.score(0)
        X = int(conn[i])
        order = [int(c3s[i][X][0]), X, int(c3s[i][X][2])]
        for nd in order:
            ot.optimize_branch(nd, 0.01)
        lens = ot.branch_lengths()[order]
        ot.make_all_dirty()
        ref.append((l0, ot.score(0), lens))
        ot.close()
    return w, c3s, dls, conn, ref


def _run(case, mixed, sequential, repeat=1):
    w, c3s, dls, conn, _ = case
    inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, len(conn), mixed=mixed)
    res = [pop.score(c3s, dls, conn, 0.01, sequential=sequential) for _ in range(repeat)]
    cnt = pop.counters()
    pop.close()
    inst.close()
    return res, cnt


def test_per_tree_plain_matches_oracle(case):
    (out, lens), = _run(case, mixed=False, sequential=True)[0]
    for i, (l0, lf, rl) in enumerate(case[4]):
        assert abs(out[i, 0] - l0) <= 1e-8 * abs(l0), (i, out[i, 0], l0)
        assert abs(out[i, 1] - lf) <= 1e-8 * abs(lf), (i, out[i, 1], lf)
        assert np.allclose(lens[i], rl, rtol=1e-6, atol=1e-10), (i, lens[i], rl)


def test_batched_plain_equals_per_tree_plain(case):
    (seq, slens), = _run(case, mixed=False, sequential=True)[0]
    (bat, blens), = _run(case, mixed=False, sequential=False)[0]
    assert np.allclose(bat[:, :2], seq[:, :2], rtol=1e-10, atol=0)
    assert np.allclose(blens, slens, rtol=1e-8, atol=1e-12)


def test_batched_precision_form_matches_oracle_and_repeats(case):
    w = case[0]
    res, cnt = _run(case, mixed=True, sequential=False, repeat=2)
    tol = 1e-4
    for out, lens in res:
        for i, (l0, lf, rl) in enumerate(case[4]):
            assert abs(out[i, 0] - l0) <= tol, (i, out[i, 0], l0)
            assert abs(out[i, 1] - lf) <= tol, (i, out[i, 1], lf)
            assert np.allclose(lens[i], rl, rtol=1e-3, atol=1e-8), (i, lens[i], rl)
    # a replay gives identical results
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    # uneven dirty sets: every candidate recomputed some CLAs, far fewer than a full tree
    ncand = len(case[3])
    per = (cnt["cla_ops"] - 3 * ncand) / ncand
    assert 1 <= per <= 60


def test_batched_precision_form_does_not_depend_on_work_item_sizes(case):
    """Tiles per item size the level and coefficient launches and the chunks
    per item the Newton sweeps' work items; every reduction has a fixed
    partition, so any choice gives bit-identical results."""
    w, c3s, dls, conn, _ = case
    inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, len(conn), mixed=True)
    runs = []
    for tiles, chunks in ((1, 1), (4, 2), (32, 4), (5, 3)):
        pop.set_tuning(tiles, chunks)
        runs.append(pop.score(c3s, dls, conn, 0.01))
    for out, lens in runs[1:]:
        assert np.array_equal(out, runs[0][0]) and np.array_equal(lens, runs[0][1])
    pop.close()
    inst.close()


def test_batched_replay_takes_the_newton_parameters_of_each_call(case):
    """The batched pass replays a captured CUDA graph when the plan repeats; a
    call with another Newton precision must run with it, exactly as a fresh
    population does."""
    w, c3s, dls, conn, _ = case
    inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, len(conn), mixed=True)
    pop.set_tuning(8, 2)
    pop.score(c3s, dls, conn, 0.01)
    again = pop.score(c3s, dls, conn, 1e-4)
    pop.close()
    inst.close()
    inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, len(conn), mixed=True)
    pop.set_tuning(8, 2)
    fresh = pop.score(c3s, dls, conn, 1e-4)
    pop.close()
    inst.close()
    assert np.array_equal(again[0], fresh[0]) and np.array_equal(again[1], fresh[1])


def test_population_switches_between_batched_and_per_tree_modes(case):
    """One precision-form population: batched (parent tree in FP64 buffers), then
    per-tree (parent rebuilt in ordinary buffers), then batched again."""
    w, c3s, dls, conn, ref = case
    inst, pop = engine.population_engine(w.data, w.child3, w.dlen, w.model, len(conn), mixed=True)
    tol = 1e-4
    runs = [pop.score(c3s, dls, conn, 0.01, sequential=s)[0] for s in (False, True, False)]
    for out in runs:
        for i, (l0, lf, _) in enumerate(ref):
            assert abs(out[i, 0] - l0) <= tol and abs(out[i, 1] - lf) <= tol
    assert np.array_equal(runs[0], runs[2])
    pop.close()
    inst.close()
