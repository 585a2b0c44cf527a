import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_fixture(name):
    """Golden fixture written by tests/golden/make_fixtures.py."""
    from garli_b200.patterns import PatternData

    with open(os.path.join(GOLDEN, name)) as f:
        fx = json.load(f)
    tips = np.array([list(bytes.fromhex(h)) for h in fx["tips_hex"]], dtype=np.uint8)
    pd = PatternData(fx["nstates"], tips, np.array(fx["counts"], dtype=np.int32), fx["last_const"],
                     np.array(fx["const_states"], dtype=np.int32), fx["nsites"])
    return fx, pd, np.array(fx["child3"], dtype=np.int32), np.array(fx["dlen"], dtype=np.float64)


def fixture_model(fx, mathlib):
    """Model of a fixture, built with ``mathlib``'s Q/eigen/gamma (oracle or engine)."""
    from garli_b200.engine import Model

    m = fx["model"]
    if fx["nstates"] == 4:
        pi = np.array(m["e"], dtype=np.float64)
        pi = pi / pi.sum()
        Q, bm = mathlib.gtr_qmat(m["r"], pi)
        rates = mathlib.discrete_gamma(m["a"], m["ncat"])
        pinv = m["p"]
        has = True
    else:
        pi = np.array(m["e_empirical"], dtype=np.float64)
        Q, bm = mathlib.codon_qmat6(m["r"], m["o"][0], pi)
        rates = np.ones(1)
        pinv, has = 0.0, False
    ev, U, Ui = mathlib.eigen(Q, pi)
    R = len(rates)
    return Model(fx["nstates"], pi, Q, bm, ev, U, Ui, np.asarray(rates, dtype=np.float64),
                 np.full(R, (1.0 - pinv) / R), pinv, has)


def fixture_params(fx, pd):
    """GARLI's model parameters of a DNA fixture: (kind, pi, rel, alpha, ncat,
    pinv, maxPinv) with maxPinv = constant sites / all sites (model.cpp:1649)."""
    m = fx["model"]
    pi = np.array(m["e"], dtype=np.float64)
    pi = pi / pi.sum()
    nconst = int(np.sum(pd.counts[: pd.last_const + 1]))
    return dict(pi=pi, rel=np.array(m["r"], dtype=np.float64), alpha=m["a"], ncat=m["ncat"], pinv=m["p"],
                max_pinv=nconst / float(np.sum(pd.counts)))


def scoring_setup(fx, pd):
    """Model parameters of a fixture and the parameters its scoring test
    estimates (tests/scoring/<conf>): n.G4 / n.G5 alpha, pinv, frequencies and
    six relative rates (mask 15); c.conf six relative rates, omega fixed,
    empirical codon frequencies (mask 8)."""
    m = fx["model"]
    if fx["nstates"] == 4:
        fp = fixture_params(fx, pd)
        return dict(kind=0, pi=fp["pi"], rel=fp["rel"], alpha=fp["alpha"], ncat=fp["ncat"], pinv=fp["pinv"],
                    max_pinv=fp["max_pinv"], omega=1.0, mask=15)
    return dict(kind=2, pi=np.array(m["e_empirical"], dtype=np.float64), rel=np.array(m["r"], dtype=np.float64),
                alpha=0.5, ncat=1, pinv=None, max_pinv=0.0, omega=m["o"][0], mask=8)


def scoring_test_score(fx, lnl, site_lnl):
    """The number the reference's scoring test compares with expected.scr
    (tests/runtests.sh): -lnL + 1/2 sum (w_c - 1) lnL_c over the weighted
    columns of the test's data file (make_fixtures.wtset_sitelike_extra)."""
    st = fx["scoring_test"]
    return -lnl + 0.5 * sum(e * site_lnl[p] for p, e in st["sitelike_extra"])


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
