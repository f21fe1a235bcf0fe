"""The C restatement of the tempered SMC sampler (oracle/gmm_oracle.c)
against vSMC's own run of the example/gmm sampler (tests/golden/gmm.npz,
made by oracle/ref_gmm.cpp): every history, particle, log-weight and engine
position bit for bit; and the product's data simulator against the
oracle's."""
import os

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("ess", "resampled", "zinc", "integrand", "grid", "accept", "params", "lw", "words")


@pytest.fixture(scope="module")
def gmm():
    return np.load(os.path.join(ROOT, "tests", "golden", "gmm.npz"))


def run_cfg(g):
    return {k: (float(g["run_" + k]) if k in ("sd", "threshold") else int(g["run_" + k]))
            for k in ("N", "iters", "power", "sweeps", "sd", "scheme", "threshold", "seed")}


def test_data_simulator(gmm):
    assert np.array_equal(O.gmm_simulate(1000, 1), gmm["data"])


def test_product_data_simulator(gmm):
    from vsmc_b200 import build as B

    if not os.path.exists(B.LIB):
        pytest.skip("libvsmc_cuda.so not built")
    from vsmc_b200 import capi

    assert np.array_equal(capi.gmm_simulate(1000, 1), gmm["data"])


def test_oracle_matches_reference_fixture(gmm):
    r = O.gmm_smc(gmm["data"], **run_cfg(gmm))
    for k in KEYS:
        assert np.array_equal(r[k], gmm[k]), k
    assert r["logz"] == float(gmm["logz"])
    assert r["path_logz"] == float(gmm["path_logz"])


@pytest.mark.skipif(not O.gmm_ref_available(), reason="reference harness not built")
@pytest.mark.parametrize("scheme,sweeps,power", [(2, 2, 2), (0, 1, 5), (4, 3, 4)])
def test_oracle_matches_reference_live(gmm, scheme, sweeps, power):
    cfg = dict(N=96, iters=16, power=power, sweeps=sweeps, sd=0.15, scheme=scheme,
               threshold=0.7, seed=7)
    a = O.gmm_smc(gmm["data"], **cfg)
    b = O.ref_gmm_smc(gmm["data"], **cfg)
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k
    assert a["logz"] == b["logz"] and a["path_logz"] == b["path_logz"]


def test_summary_table_fixture(gmm):
    """gmm_summary.tsv is the table of the fixture's own run."""
    rows = open(os.path.join(ROOT, "tests", "golden", "gmm_summary.tsv")).read().splitlines()
    head = rows[0].split("\t")
    assert head[:2] == ["Size", "Resampled"] and head[-4:] == ["ESS", "Path.Integrand",
                                                              "Path.Grid", ""]
    body = [r.split("\t")[:-1] for r in rows[1:]]
    assert len(body) == int(gmm["run_iters"]) + 1
    for t, cols in enumerate(body):
        assert int(cols[1]) == int(gmm["resampled"][t])
        assert [int(c) for c in cols[2:18]] == list(gmm["accept"][t])
        assert float(cols[18]) == float("%g" % gmm["ess"][t])
