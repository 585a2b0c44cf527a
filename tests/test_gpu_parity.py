"""Parity of the CUDA engine with the CPU oracle, through the C ABI (needs a B200).

Tolerances:
  * plain FP64 form: lnL, d1, d2 to 1e-8 relative (|dlnL| <= 1e-8 |lnL|); CLA
    entries to 1e-12 (4 states) / 1e-9 (61 states) of each pattern's largest
    entry (P(t) uses the device exp, which may differ from the host's by an
    ulp); integer rescale counts and ranks exactly.
  * precision form (FP32 CLAs, power-of-two scalers): |dlnL| <= 1e-4
    absolute per tree, derivatives to 1e-4 relative.
"""
import numpy as np
import pytest

from conftest import fixture_model, load_fixture
from garli_b200 import engine, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

PINS = ["z11x2178_nG4.json", "z11x2178_nG5.json", "z11x2178_codon.json"]


@pytest.fixture(scope="module", autouse=True)
def _device():
    if engine.lib().gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")


def _both(pd, c3, dl, model, mixed=False, omodel=None):
    """Engine and oracle on the same tree; ``omodel`` is the same model built
    with the oracle's own model math (default: ``model`` itself)."""
    inst, tree = engine.tree_engine(pd, c3, dl, model, mixed=mixed)
    ot = orc.OracleTree(pd, c3, dl, model if omodel is None else omodel)
    return inst, tree, ot


@pytest.mark.parametrize("name", PINS)
def test_fixture_scores_match_oracle_and_garli(name):
    fx, pd, c3, dl = load_fixture(name)
    m = fixture_model(fx, engine)
    inst, tree, ot = _both(pd, c3, dl, m, omodel=fixture_model(fx, orc))
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-8 * abs(lo)
    assert abs(lg - fx["garli_score"]) < 2e-6
    assert np.allclose(inst.site_lnl(), ot.site_lnl(), rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("name", PINS)
def test_every_cla_and_scaler_matches(name):
    """After a full score from node 0 every clean CLA equals the oracle's; scalers
    exactly.  Both sides take the same eigensystem here, so the comparison is of
    the CLA arithmetic alone (the model math is compared in the score tests)."""
    fx, pd, c3, dl = load_fixture(name)
    m = fixture_model(fx, engine)
    inst, tree, ot = _both(pd, c3, dl, m)
    for tr in (tree, ot):
        tr.rescale_every = 2  # force rescaling on every eligible CLA
        tr.score(0)
    n = 0
    for nd in [0] + list(range(pd.ntax + 1, c3.shape[0])):
        for w in range(3):
            b = tree.cla_buffer(nd, w)
            arr, mult = ot.cla(nd, w)
            assert (b >= 0) == (arr is not None)
            if b < 0:
                continue
            g = inst.partials(b)
            # normwise per pattern: 61-state P(t) sums cancel, so entries far below a
            # pattern's largest carry the ulp-level exp differences of host vs device
            tol = 1e-12 if pd.nstates == 4 else 1e-9
            scale = np.abs(arr).max(axis=(1, 2), keepdims=True)
            assert (np.abs(g - arr) <= tol * scale).all(), (nd, w, np.abs(g - arr).max())
            assert np.array_equal(inst.scale_factors(b), mult)
            assert engine.lib().gb_get_rescale_rank(inst.h, b) == ot.cla_rank(nd, w)
            n += 1
    assert n >= pd.ntax - 2


@pytest.mark.parametrize("name", PINS)
def test_branch_derivatives(name):
    """d1 near an optimum is a small sum of large terms of both signs: the same
    eigensystem on both sides keeps the comparison to the derivative arithmetic."""
    fx, pd, c3, dl = load_fixture(name)
    m = fixture_model(fx, engine)
    inst, tree, ot = _both(pd, c3, dl, m)
    for nd in range(1, c3.shape[0]):
        g = tree.derivatives(nd)
        o = ot.derivatives(nd)
        assert abs(g[0] - o[0]) <= 1e-8 * abs(o[0])
        assert abs(g[1] - o[1]) <= 1e-8 * max(1.0, abs(o[1])), (nd, g, o)
        assert abs(g[2] - o[2]) <= 1e-8 * max(1.0, abs(o[2])), (nd, g, o)


def test_root_choice_and_rescale_invariance():
    fx, pd, c3, dl = load_fixture(PINS[0])
    m = fixture_model(fx, engine)
    inst, tree, ot = _both(pd, c3, dl, m, omodel=fixture_model(fx, orc))
    ref = ot.score(0)
    for nd in [0] + list(range(pd.ntax + 1, c3.shape[0])):
        tree.make_all_dirty()
        assert abs(tree.score(nd) - ref) <= 1e-8 * abs(ref)
    tree.rescale_every = 2
    tree.make_all_dirty()
    assert abs(tree.score(0) - ref) <= 1e-8 * abs(ref)


def test_small_tree_score_and_newton_pass():
    """32 taxa x 2,000 sites GTR+G4: full score plus one all-branch Newton pass."""
    w = synth.dna_small()
    inst, tree, ot = _both(w.data, w.child3, w.dlen, w.model, omodel=w.model_with(orc))
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-8 * abs(lo)
    ig, fg = tree.optimize_all_branches(0.01)
    io, fo = ot.optimize_all_branches(0.01)
    assert abs(fg - fo) <= 1e-8 * abs(fo)
    assert np.allclose(tree.branch_lengths(), ot.branch_lengths(), rtol=1e-6, atol=1e-10)
    tree.make_all_dirty()
    ot.make_all_dirty()
    assert abs(tree.score(0) - ot.score(0)) <= 1e-8 * abs(lo)


def _underflowing_case(seed=11, ntax=96, nsites=300, blen=1e-5):
    """Random tip states on short branches: every site needs many substitutions, so
    site likelihoods fall by ~1e-3 per mismatch and cross 1e-190 within one
    rescale window unless rescaleEvery is small."""
    from garli_b200.patterns import compress

    rng = np.random.default_rng(seed)
    c3, dl = synth.yule_tree(ntax, rng, 0.1)
    dl[:] = blen
    dl[0] = 0.0
    m = synth.gtr_model(rng)
    states = rng.integers(4, size=(ntax, nsites))
    return c3, dl, m, compress(synth.dna_to_masks(states), 4)


def test_rescale_retry_path_matches_oracle():
    """GARLI's throw(1) -> rescaleEvery -= 2 retry (tree.cpp:3442, :4077)."""
    c3, dl, m, pd = _underflowing_case()
    inst, tree, ot = _both(pd, c3, dl, m)
    for tr in (tree, ot):
        tr.rescale_every = 160
    lo = ot.score(0)
    lg = tree.score(0)
    assert ot.rescale_every < 160, "case did not trigger the retry path"
    assert tree.rescale_every == ot.rescale_every
    assert tree.counters()["rescale_retries"] == (160 - ot.rescale_every) // 2
    assert abs(lg - lo) <= 1e-8 * abs(lo)


@pytest.mark.parametrize("kind", ["aa", "codon"])
def test_nstate_synthetic(kind):
    w = synth.aa(seed=4, ntax=16, nsites=600) if kind == "aa" else synth.codon(seed=5, ntax=12, ncodons=300)
    inst, tree, ot = _both(w.data, w.child3, w.dlen, w.model, omodel=w.model_with(orc))
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-8 * abs(lo)
    for nd in (1, 5, w.data.ntax + 2):
        g, o = tree.derivatives(nd), ot.derivatives(nd)
        assert np.allclose(g, o, rtol=1e-8, atol=1e-8)


@pytest.mark.parametrize("ncat", [1, 3, 8])
def test_nstate_category_counts(ncat):
    """20 states with 1, 3 and 8 rate categories: the CUDA-core CLA kernel's
    tile holds one warp task per (category, 16 patterns), so the category
    count sets the tile (64, 32, 16 patterns) and the idle warps.  Plain form
    against the oracle at 1e-8, precision form (CUDA cores) at 1e-4."""
    rng = np.random.default_rng(40 + ncat)
    c3, dl = synth.yule_tree(14, rng, 0.15)
    spec = synth.aa_spec(rng, 0.7, ncat)
    m = synth.build_model(spec)
    w = synth.Workload(f"aa_{ncat}", c3, dl, m, synth.compress(synth.simulate(c3, dl, m, 700, rng), 20), spec)
    inst, tree, ot = _both(w.data, c3, dl, m, omodel=w.model_with(orc))
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-8 * abs(lo)
    for nd in (1, w.data.ntax + 2):
        assert np.allclose(tree.derivatives(nd), ot.derivatives(nd), rtol=1e-8, atol=1e-8)
    tree.close()
    inst.close()
    inst, tree = engine.tree_engine(w.data, c3, dl, m, mixed=True)
    inst.set_tensor_cores(False)
    assert abs(tree.score(0) - lo) <= 1e-4
    tree.close()
    inst.close()


def test_codon_two_categories():
    """61 states with 2 rate categories: the edge kernel's matrices (P, dP,
    d2P: 179 KB) fill most of shared memory and the tiles shrink to one warp
    task per category.  Plain form against the oracle at 1e-8."""
    rng = np.random.default_rng(61)
    c3, dl = synth.yule_tree(10, rng, 0.2)
    base = synth.codon_spec(rng)
    spec = synth.ModelSpec("codon", base.pi, None, 0.6, 2, None, base.kappa, base.omega)
    m = synth.build_model(spec)
    w = synth.Workload("codon_2", c3, dl, m, synth.compress(synth.simulate(c3, dl, m, 300, rng), 61), spec)
    inst, tree, ot = _both(w.data, c3, dl, m, omodel=w.model_with(orc))
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-8 * abs(lo)
    for nd in (1, w.data.ntax + 2):
        assert np.allclose(tree.derivatives(nd), ot.derivatives(nd), rtol=1e-8, atol=1e-8)
    tree.close()
    inst.close()


@pytest.mark.parametrize("name", PINS)
def test_mixed_precision_form(name):
    fx, pd, c3, dl = load_fixture(name)
    m = fixture_model(fx, engine)
    inst, tree = engine.tree_engine(pd, c3, dl, m, mixed=True)
    ot = orc.OracleTree(pd, c3, dl, fixture_model(fx, orc))
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-4
    for nd in (1, 4, pd.ntax + 3):
        g, o = tree.derivatives(nd), ot.derivatives(nd)
        assert abs(g[0] - o[0]) <= 1e-4
        assert abs(g[1] - o[1]) <= 1e-4 * max(1.0, abs(o[1]))
        assert abs(g[2] - o[2]) <= 1e-4 * max(1.0, abs(o[2]))


def test_abi_operation_lists_directly():
    """Drive the instance ABI with hand-built ClaOperation lists (tip-tip, int-tip, int-int)."""
    w = synth.make_dna(6, 400, seed=3)
    pd, c3, dl, m = w.data, w.child3, w.dlen, w.model
    ntip = 6
    inst = engine.Instance(ntip, 12, 4, pd.npat, 4, 10)
    inst.set_data(pd)
    inst.set_model(m)
    inst.update_transition_matrices([(i, dl[i], 0, 1) for i in range(1, 10)])
    ot = orc.OracleTree(pd, c3, dl, m)
    lo = ot.score(0)

    def buf(nd):  # tips 1..6 -> 0..5; internal 0, 7, 8, 9 -> 6..9
        return nd - 1 if 1 <= nd <= ntip else ntip + (0 if nd == 0 else nd - ntip)

    level = {}
    ops = []

    def post(nd):
        l, r = int(c3[nd][0]), int(c3[nd][2])
        if nd == 0 and c3[0][1] > ntip:
            post(int(c3[0][1]))
        for k in (l, r):
            if k > ntip:
                post(k)
        lvl = 1 + max([level[k] for k in (l, r) if k > ntip] or [0])
        level[nd] = lvl
        ops.append((buf(nd), buf(l), buf(r), l, r, lvl))

    post(0)
    inst.update_partials(ops, 16)
    mid = int(c3[0][1])
    out = inst.calculate_edge(buf(0), buf(mid), mid, derivatives=False)
    assert abs(out[0] - lo) <= 1e-8 * abs(lo)
    assert inst.launch_count() > 0


@pytest.mark.parametrize("mixed", [False, True])
def test_device_newton_pass_equals_host_pass(mixed):
    """The graph pass takes exactly the host driver's Newton decisions (same
    partition of the pattern sums, same gb::nr_step); so does the persistent
    pass of the plain form.  The precision form's persistent pass has its own
    fused arithmetic (k_pass4m): there the optimised lengths agree to 1e-3
    relative and the rescored lnL to the precision form's bar."""
    w = synth.make_dna(40, 3000, seed=21, pinv_range=(0.05, 0.3))
    res = {}
    for mode in ("persistent", "graph", "host"):
        inst, tree = engine.tree_engine(w.data, w.child3, w.dlen * 1.3, w.model, mixed=mixed)
        inst.set_pass_mode(mode == "persistent")
        tree.set_device_newton(mode != "host")
        tree.score(0)
        imp, _ = tree.optimize_all_branches(0.01)
        bl = tree.branch_lengths()
        tree.make_all_dirty()
        res[mode] = (bl, tree.score(0), imp)
        tree.close()
        inst.close()
    exact = ["graph", "persistent"] if not mixed else ["graph"]
    for m in exact:
        bl, lnl, imp = res[m]
        assert np.array_equal(res["host"][0], bl), (m, np.abs(res["host"][0] - bl).max())
        assert res["host"][1] == lnl and res["host"][2] == imp
    if mixed:
        bl, lnl, imp = res["persistent"]
        assert np.allclose(bl, res["host"][0], rtol=1e-3, atol=1e-8)
        assert abs(lnl - res["host"][1]) <= 1e-4


def test_device_newton_pass_matches_oracle_and_is_repeatable():
    w = synth.make_dna(48, 2500, seed=22)
    inst, tree, ot = _both(w.data, w.child3, w.dlen * 0.7, w.model, omodel=w.model_with(orc))
    for _ in range(2):  # second pass replays the cached graph from a different start
        tree.score(0)
        ot.score(0)
        tree.optimize_all_branches(0.01)
        ot.optimize_all_branches(0.01)
        assert np.allclose(tree.branch_lengths(), ot.branch_lengths(), rtol=1e-6, atol=1e-10)
        tree.make_all_dirty()
        ot.make_all_dirty()
        lg, lo = tree.score(0), ot.score(0)
        assert abs(lg - lo) <= 1e-8 * abs(lo)


def test_device_newton_pass_rescale_retry():
    """A pass whose CLAs cross the bail-out is rerun with a lower rescaleEvery."""
    c3, dl, m, pd = _underflowing_case(ntax=64, nsites=200)
    inst, tree, ot = _both(pd, c3, dl, m)
    tree.rescale_every = 120
    tree.score(0)
    tree.optimize_all_branches(0.01)
    assert tree.counters()["rescale_retries"] > 0
    bl = tree.branch_lengths()
    for nd in range(1, len(bl)):
        ot.set_branch_length(nd, bl[nd])
    tree.make_all_dirty()
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-8 * abs(lo)


@pytest.mark.parametrize("kind,mixed", [("dna", False), ("dna", True), ("aa", False), ("codon", True)])
def test_site_derivatives(kind, mixed):
    """gb_get_site_derivatives (beagleGetSiteDerivatives): the per-pattern d1,
    d2 of a derivative evaluation, weighted by the pattern counts, sum to the
    evaluation's d1, d2, and the site lnLs to its lnL (1e-9 relative); a
    score-only evaluation leaves no site derivatives to read."""
    w = {"dna": lambda: synth.make_dna(24, 1500, 7, pinv_range=(0.05, 0.3)),
         "aa": lambda: synth.aa(ntax=12, nsites=400), "codon": lambda: synth.codon(ntax=10, ncodons=200)}[kind]()
    inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model, mixed=mixed)
    tree.score(0)
    with pytest.raises(engine.EngineError):
        inst.site_derivatives()
    cnt = np.asarray(w.data.counts, dtype=np.float64)
    for nd in (1, w.data.ntax + 2, w.child3.shape[0] - 1):
        lnl, d1, d2 = tree.derivatives(nd)
        s1, s2 = inst.site_derivatives()
        u = inst.site_lnl()
        keep = u < 0.0  # the n-state kernels drop non-negative site lnLs, as GARLI does
        assert abs(np.sum(cnt[keep] * u[keep]) - lnl) <= 1e-9 * abs(lnl)
        assert abs(np.sum(cnt[keep] * s1[keep]) - d1) <= 1e-9 * max(1.0, abs(d1)), (nd, d1)
        assert abs(np.sum(cnt[keep] * s2[keep]) - d2) <= 1e-9 * max(1.0, abs(d2)), (nd, d2)
    tree.close()
    inst.close()
