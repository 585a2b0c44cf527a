"""The device eigensolver (gb_set_eigen_from_rate_matrices, Model::CalcEigenStuff
model.cpp:827-856 on the GPU) against the host one GARLI's tree layer uses.

Eigen-decompositions differ in eigenvalue order and eigenvector signs, so they
are compared through what they feed: P(t), dP/dt, d2P/dt2 at several lengths
(to 1e-12 of the largest entry), then through a full plain-FP64 score against
the oracle (1e-8 relative).
"""
import numpy as np
import pytest

from garli_b200 import engine, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _models():
    rng = np.random.default_rng(17)
    return {"gtr": synth.gtr_model(rng, 0.5, 4, 0.2), "aa": synth.aa_model(rng), "codon": synth.codon_model(rng)}


@pytest.mark.parametrize("kind", ["gtr", "aa", "codon"])
def test_device_eigensystem_gives_host_transition_matrices(kind):
    if engine.lib().gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")
    m = _models()[kind]
    S, R = m.nstates, m.ncat
    inst = engine.Instance(4, 4, S, 100, R, 8, neigen=2)
    inst.set_model(m, eigen_index=0)  # host eigensystem in slot 0
    sw = inst.set_eigen_from_q([1], m.Q.reshape(1, S, S), m.pi.reshape(1, S), [m.blen_mult])
    assert 0 < sw[0] < 40
    lens = [1e-6, 0.01, 0.1, 0.7, 3.0]
    ops = [(i, t, 0, 1) for i, t in enumerate(lens)] + [(len(lens) + i, t, 1, 1) for i, t in enumerate(lens[:3])]
    inst.update_transition_matrices(ops)
    for i in range(3):
        for which in range(3):
            a = inst.transition_matrix(i, which)
            b = inst.transition_matrix(len(lens) + i, which)
            assert np.allclose(a, b, rtol=0, atol=1e-12 * max(1.0, np.abs(a).max())), (kind, i, which)
    inst.close()


def test_batched_eigensystems_score_like_the_oracle():
    if engine.lib().gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")
    w = synth.make_dna(20, 800, seed=5, pinv_range=(0.05, 0.3))
    inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model)
    ot = orc.OracleTree(w.data, w.child3, w.dlen, w.model_with(orc))
    m = w.model
    # three models in one launch; slot 0 (the tree's) is replaced by the device result
    rng = np.random.default_rng(3)
    others = [synth.gtr_model(rng) for _ in range(2)]
    Qs = np.stack([m.Q] + [o.Q for o in others])
    pis = np.stack([m.pi] + [o.pi for o in others])
    with pytest.raises(engine.EngineError):
        inst.set_eigen_from_q([0, 1, 2], Qs, pis, [m.blen_mult] * 3)  # the instance has one eigen slot
    inst.set_eigen_from_q([0], Qs[:1], pis[:1], [m.blen_mult])
    tree.make_all_dirty()
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= 1e-8 * abs(lo)
    tree.close()
    inst.close()
