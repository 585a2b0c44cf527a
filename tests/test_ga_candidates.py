"""Host logic of the GA-population workload: SPR/NNI candidates of a base tree
(Tree::SPRMutate, tree.cpp:3148-3248) in GARLI's layout on the base node numbers."""
import numpy as np
import pytest

from garli_b200 import synth
from oracle import oracle as orc


def _parents(c3):
    par = {}
    for v in range(c3.shape[0]):
        for c in c3[v]:
            if c >= 0:
                assert int(c) not in par
                par[int(c)] = v
    return par


@pytest.mark.parametrize("radius", [1, 2, 5, 8])
def test_spr_move_gives_a_valid_tree(radius):
    rng = np.random.default_rng(radius)
    c3, dl = synth.yule_tree(40, rng, 0.1)
    n3, nd, P = synth.spr_move(c3, dl, rng, radius)
    par = _parents(n3)
    assert len(par) == n3.shape[0] - 1 and 0 not in par
    assert n3[0][1] >= 0 and all(n3[t].max() < 0 for t in range(1, 41))
    assert 41 <= P < n3.shape[0] and n3[P][1] == -1
    # total length kept up to the min_brlen clamp of the halved branch
    assert abs(nd.sum() - dl.sum()) < 1e-12 + 2 * synth.MIN_BRLEN
    # the tree changed: some taxon bipartition differs
    assert not np.array_equal(n3, c3)


def test_nni_is_radius_one_and_keeps_the_likelihood_of_an_unchanged_split():
    w = synth.make_dna(12, 300, seed=5)
    c3s, dls, conn = synth.ga_candidates(w.child3, w.dlen, 6, seed=9, radius_range=(1, 1))
    base = orc.OracleTree(w.data, w.child3, w.dlen, w.model)
    lb = base.score(0)
    for i in range(len(conn)):
        ot = orc.OracleTree(w.data, c3s[i], dls[i], w.model)
        li = ot.score(0)
        assert np.isfinite(li) and li != lb
        # root invariance on the candidate (Population::RunTests)
        X = int(conn[i])
        assert abs(ot.score(X) - li) < 1e-6 * abs(li)
        ot.close()
    base.close()
