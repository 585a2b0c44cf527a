"""gb_edge_loglik_static, the edge evaluation that allocates no device memory.

Some callers of the engine cannot call cudaMalloc: plugins inside a host
application that owns every device allocation through its own pool, and code
on a latency-critical thread that must not take cudaMalloc's implicit device
synchronisation.  They evaluate a branch with
gb_edge_loglik_static on device arrays they already hold; the entry point keeps
its per-block partial sums in a fixed array inside the library.  Here its lnL,
d1 and d2 must equal those of the instance path (gb_calculate_edge, reached
through Tree::CalcDerivativesRateHet) to the plain FP64 form's bar of 1e-8
relative, on two calls in a row: the second call reuses the array the first one
left behind.  The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from garli_b200 import engine, synth

pytestmark = pytest.mark.gpu

RTOL = 1e-8


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _static_edge(torch, L, inst, pd, model, nd, pbuf, child_is_tip, cbuf, derivs):
    partial = _dev(inst.partials(pbuf), torch)
    pscal = _dev(inst.scale_factors(pbuf), torch)
    if child_is_tip:
        child, cscal = None, None
        tips = _dev(pd.tips[nd - 1].astype(np.uint8), torch)
    else:
        child = _dev(inst.partials(cbuf), torch)
        cscal = _dev(inst.scale_factors(cbuf), torch)
        tips = None
    mats = _dev(np.concatenate([inst.transition_matrix(nd, k).ravel() for k in range(3)]), torch)
    freqs = _dev(np.asarray(model.pi, dtype=np.float64), torch)
    weights = _dev(np.asarray(model.probs, dtype=np.float64), torch)
    counts = _dev(pd.counts.astype(np.int32), torch)
    cs = np.full(pd.npat, -1, dtype=np.int32)
    cs[: pd.last_const + 1] = pd.const_states[: pd.last_const + 1]
    cstates = _dev(cs, torch)
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream(0).cuda_stream
    rc = L.gb_edge_loglik_static(0, model.ncat, pd.npat, _ptr(partial), _ptr(pscal), _ptr(child), _ptr(cscal),
                                 _ptr(tips), _ptr(mats), _ptr(freqs), _ptr(weights), _ptr(counts), _ptr(cstates),
                                 float(model.pinv), int(model.has_pinv), int(derivs), C.c_void_p(stream),
                                 _ptr(out))
    assert rc == 0, (rc, L.gb_last_error())
    torch.cuda.synchronize(0)
    return out.cpu().numpy()


def test_static_edge_matches_instance_edge_twice():
    torch = pytest.importorskip("torch")
    L = engine.lib()
    if L.gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")
    w = synth.make_dna(24, 3000, seed=31, pinv_range=(0.05, 0.3))
    pd, c3 = w.data, w.child3
    inst, tree = engine.tree_engine(pd, c3, w.dlen, w.model)  # plain FP64 form
    tree.score(0)
    anc = {int(k): n for n in range(c3.shape[0]) for k in c3[n] if k >= 0}
    internal = next(n for n in range(pd.ntax + 1, c3.shape[0]) if n in anc)
    for nd in (internal, 1):
        ref = np.asarray(tree.derivatives(nd))  # gb_calculate_edge through the tree layer
        a = anc[nd]
        which = 1 if c3[a][0] == nd else 2 if c3[a][2] == nd else 0
        pbuf = tree.cla_buffer(a, which)
        tip = nd <= pd.ntax
        cbuf = -1 if tip else tree.cla_buffer(nd, 0)
        assert pbuf >= 0 and (tip or cbuf >= 0)
        for _ in range(2):
            got = _static_edge(torch, L, inst, pd, w.model, nd, pbuf, tip, cbuf, derivs=True)
            assert np.all(np.isfinite(got))
            assert np.allclose(got, ref, rtol=RTOL, atol=RTOL * abs(ref[0])), (nd, got, ref)
        # lnL only: d1 = d2 = 0, lnL unchanged
        got = _static_edge(torch, L, inst, pd, w.model, nd, pbuf, tip, cbuf, derivs=False)
        assert abs(got[0] - ref[0]) <= RTOL * abs(ref[0]) and got[1] == 0.0 and got[2] == 0.0
    tree.close()
    inst.close()


def test_static_edge_rejects_sizes_beyond_its_array():
    L = engine.lib()
    if L.gb_get_device_count() < 1:
        pytest.fail("no CUDA device visible to the engine")
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.gb_edge_loglik_static(0, 4, (1 << 22) + 1, dummy, dummy, dummy, dummy, None, dummy, dummy, dummy, dummy,
                                 None, 0.0, 0, 1, None, dummy)
    assert rc == -5
    assert b"GB_STATIC_EDGE_MAX_PATTERNS" in L.gb_last_error()
