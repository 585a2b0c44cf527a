"""CLA launch shapes chosen by timing (needs a B200).

gb_set_cla_tuning / the autotuner pick the blocks per SM of the per-tree
precision 4-state level launch and the patterns per block of the n-state
CUDA-core kernel.  Each pattern's arithmetic does not depend on the shape, so
every choice must give the same bits: scores, derivatives, CLAs and scalers
are compared for equality across explicit choices and the autotuned one.
"""
import numpy as np
import pytest

from garli_b200 import engine, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    if engine.lib().gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")


def _run(w, mixed, tuning, tc=None):
    inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model, mixed=mixed)
    if tc is not None:
        inst.set_tensor_cores(tc)
    if tuning is not None:
        inst.set_cla_tuning(*tuning)
    lnl = tree.score(0)
    d = tree.derivatives(w.data.ntax + 2)
    nn = w.child3.shape[0]
    clas = {}
    for nd in (0, w.data.ntax + 1, nn - 1):
        b = tree.cla_buffer(nd, 0)
        if b >= 0:
            clas[nd] = (inst.partials(b), inst.scale_factors(b))
    state = inst.cla_tuning()
    tree.close()
    inst.close()
    return lnl, d, clas, state


def _same(a, b):
    assert a[0] == b[0], (a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert a[2].keys() == b[2].keys()
    for nd in a[2]:
        assert np.array_equal(a[2][nd][0], b[2][nd][0]), nd
        assert np.array_equal(a[2][nd][1], b[2][nd][1]), nd


def test_level_shape_choices_agree():
    w = synth.make_dna(64, 40000, 11, pinv_range=(0.05, 0.3))  # 62 updates x ~27k patterns: tuned
    ref = _run(w, True, (4, -1))
    assert not ref[3]["pending"] and ref[3]["level_blocks_per_sm"] == 4
    for t in ((32, -1), (8, -1)):
        _same(_run(w, True, t), ref)
    auto = _run(w, True, None)
    assert not auto[3]["pending"] and auto[3]["level_blocks_per_sm"] in (4, 8, 16, 32)
    _same(auto, ref)


@pytest.mark.parametrize("mixed", [False, True])
def test_nstate_tile_choices_agree(mixed):
    w = synth.aa(ntax=48, nsites=12000)
    ref = _run(w, mixed, (-1, 16), tc=False)
    assert ref[3]["nstate_tile"] == 16
    rounded = _run(w, mixed, (-1, 24), tc=False)  # rounded up to the 16-pattern warp task
    assert rounded[3]["nstate_tile"] == 32
    _same(rounded, ref)
    _same(_run(w, mixed, (-1, 64), tc=False), ref)
    auto = _run(w, mixed, None, tc=False)
    _same(auto, ref)
