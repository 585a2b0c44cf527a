"""The tensor-core CLA update of the precision form (20 and 61 states).

k_cla_i8 computes each P.CLA product on the tensor cores from base-256 digit
splits of the CLA and of P(t) (tcgen05.mma kind::i8, exact 32-bit integer
accumulation), bounded by (2^-38 + 2^-38 S + 2^-34 S) of the CLA row's
largest entry.  Checked against the CUDA-core precision kernel (FP64
arithmetic on the same FP32 CLAs) and the FP64 oracle.

Tolerances: every CLA entry, taken with its pattern's power-of-two scaler
(the two kernels pick different powers of two), within 2e-5 of the pattern's
largest entry against the CUDA-core kernel, median over patterns within 1e-6
(FP32-level agreement that grows with the depth of the CLA: both paths round
every level to FP32 independently); lnL, d1, d2 as the precision form's bar:
|dlnL| <= 1e-4 absolute, derivatives 1e-4 relative to max(1, |d|).
"""
import numpy as np
import pytest

from garli_b200 import engine, synth
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _workload(kind):
    if kind == "aa":
        return synth.aa(seed=6, ntax=24, nsites=3000)
    return synth.codon(seed=7, ntax=16, ncodons=1500)


@pytest.mark.parametrize("kind", ["aa", "codon"])
def test_tensor_core_clas_match_cuda_core_clas(kind):
    w = _workload(kind)
    res = []
    for tc in (True, False):
        inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model, mixed=True)
        inst.set_tensor_cores(tc)
        tree.score(0)
        clas = {}
        for nd in [0] + list(range(w.data.ntax + 1, w.child3.shape[0])):
            for wh in range(3):
                b = tree.cla_buffer(nd, wh)
                if b >= 0:
                    clas[(nd, wh)] = (inst.partials(b), inst.scale_factors(b))
        res.append(clas)
        tree.close()
        inst.close()
    assert res[0].keys() == res[1].keys() and len(res[0]) > 0
    for k in res[0]:
        (a, sa), (b, sb) = res[0][k], res[1][k]
        # the CLA's value is the stored one times 2^-scaler
        a = a * np.exp2(-sa.astype(np.float64))[:, None, None]
        b = b * np.exp2(-sb.astype(np.float64))[:, None, None]
        mx = b.reshape(b.shape[0], -1).max(axis=1)
        err = np.abs(a - b).reshape(a.shape[0], -1).max(axis=1) / mx
        assert err.max() <= 2e-5 and np.median(err) <= 1e-6, (k, err.max(), np.median(err))


@pytest.mark.parametrize("kind", ["aa", "codon"])
def test_tensor_core_precision_form_matches_oracle(kind):
    w = _workload(kind)
    inst, tree = engine.tree_engine(w.data, w.child3, w.dlen, w.model, mixed=True)
    ot = orc.OracleTree(w.data, w.child3, w.dlen, w.model_with(orc))
    tol = 1e-4
    lg, lo = tree.score(0), ot.score(0)
    assert abs(lg - lo) <= tol, (lg, lo)
    for nd in (1, 3, w.data.ntax + 2):
        g, o = tree.derivatives(nd), ot.derivatives(nd)
        assert abs(g[0] - o[0]) <= tol
        assert abs(g[1] - o[1]) <= 1e-4 * max(1.0, abs(o[1]))
        assert abs(g[2] - o[2]) <= 1e-4 * max(1.0, abs(o[2]))
    tree.close()
    inst.close()
