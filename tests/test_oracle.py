"""The C restatement (oracle/smc_oracle.c) against the fixtures generated from
the unmodified vSMC headers: every comparison is bit-exact, which pins the
oracle that the CUDA path is later checked against."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("i", range(4))
def test_philox_words(golden, i):
    k, c = golden[f"philox_{i}_key"], golden[f"philox_{i}_ctr"]
    s = int(golden[f"philox_{i}_skip"])
    ref = golden[f"philox_{i}_words"]
    assert np.array_equal(O.philox_stream(k, c, ref.size, s), ref)


@pytest.mark.parametrize("i", range(4))
def test_threefry_words(golden, i):
    k, c = golden[f"threefry_{i}_key"], golden[f"threefry_{i}_ctr"]
    s = int(golden[f"threefry_{i}_skip"])
    ref = golden[f"threefry_{i}_words"]
    assert np.array_equal(O.threefry_stream(k, c, ref.size, s), ref)


def test_canonical_edges():
    # generate_canonical clamps a rounded-up 1.0 to the largest double below 1
    assert O.canonical_u64(2**64 - 1) == np.nextafter(1.0, 0.0)
    assert O.canonical_u64(0) == 0.0
    assert O.canonical_u64(1 << 63) == 0.5
    assert O.canonical_u32x2(0xFFFFFFFF, 0xFFFFFFFF) == np.nextafter(1.0, 0.0)
    assert O.canonical_u32x2(0, 1 << 31) == 0.5


@pytest.mark.parametrize("i", range(3))
def test_weight_set(golden, i):
    ess, w, lw = O.add_log_weight(golden[f"weight_{i}_lw"], golden[f"weight_{i}_inc"])
    assert ess == golden[f"weight_{i}_ess"]
    assert np.array_equal(w, golden[f"weight_{i}_w"])
    assert np.array_equal(lw, golden[f"weight_{i}_lwout"])


def _res_cases(golden):
    for name in golden["res_names"]:
        for sch in range(6):
            for seed, skip in ((103, 0), (7, 5)):
                yield str(name), sch, seed, skip


def test_resample_all(golden):
    n = 0
    for name, sch, seed, skip in _res_cases(golden):
        w = golden[f"res_{name}_w"]
        N = int(golden[f"res_{name}_N"])
        tag = f"res_{name}_s{sch}_{seed}_{skip}"
        rep, cf, words = O.resample(sch, w, seed, skip, M=w.size, N=N)
        assert np.array_equal(rep, golden[tag + "_rep"]), tag
        assert words == int(golden[tag + "_words"]), tag
        if N == w.size:
            assert np.array_equal(cf, golden[tag + "_cf"]), tag
        n += 1
    assert n > 100


def test_cfrp_invariants(golden):
    """cfrp_trans keeps survivors in place and sources only survivors."""
    for name, sch, seed, skip in _res_cases(golden):
        w = golden[f"res_{name}_w"]
        if int(golden[f"res_{name}_N"]) != w.size:
            continue
        tag = f"res_{name}_s{sch}_{seed}_{skip}"
        rep, cf = golden[tag + "_rep"], golden[tag + "_cf"]
        assert rep.sum() == w.size
        idx = np.arange(w.size)
        assert np.array_equal(cf[rep > 0], idx[rep > 0])
        assert np.all(rep[cf] > 0)
        assert np.array_equal(np.bincount(cf, minlength=w.size), rep)


@pytest.mark.parametrize("sch", range(6))
def test_cv_filter(golden, sch):
    ox, oy = golden["cv_obs_x"], golden["cv_obs_y"]
    r = O.cv_filter(1000, 100, sch, ox, oy, seed=101, want_state=(sch == 0))
    assert r["logz"] == golden[f"cv_s{sch}_logz"]
    for k in ("ess", "resampled", "logz_inc", "mean_x", "mean_y"):
        assert np.array_equal(r[k], golden[f"cv_s{sch}_{k}"]), k
    assert r["words_used"] == int(golden[f"cv_s{sch}_words"])
    if sch == 0:
        assert np.array_equal(r["state"], golden["cv_s0_state"])
        assert np.array_equal(r["lw"], golden["cv_s0_lw"])


def test_cv_filter_stream(golden):
    ox, oy = O.cv_simulate(30, obs_seed=11, stream=3)
    assert np.array_equal(ox, golden["cv2_obs_x"]) and np.array_equal(oy, golden["cv2_obs_y"])
    r = O.cv_filter(4096, 30, 3, ox, oy, seed=5, stream=3, threshold=0.8)
    assert r["logz"] == golden["cv2_logz"]
    for k in ("ess", "resampled", "logz_inc", "mean_x", "mean_y"):
        assert np.array_equal(r[k], golden[f"cv2_{k}"]), k


def test_simulated_observations(golden):
    ox, oy = O.cv_simulate(100, obs_seed=7)
    assert np.array_equal(ox, golden["cv_obs_x"])
    assert np.array_equal(oy, golden["cv_obs_y"])


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_reference_backends_agree():
    """StateOMP, StateSTD and StateSEQ give byte-identical filters (the
    reference's cross-backend property) and equal the oracle."""
    ox, oy = O.cv_simulate(20, obs_seed=3)
    rs = [O.ref_cv_filter(512, 20, 0, ox, oy, seed=9, backend=b) for b in (0, 1, 2)]
    ro = O.cv_filter(512, 20, 0, ox, oy, seed=9)
    for r in rs:
        assert r["logz"] == ro["logz"]
        assert np.array_equal(r["mean_x"], ro["mean_x"])


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_prospective_golden_matches_reference():
    """tests/golden/prospective.npz is what the vSMC build here gives."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "prospective.npz"))
    rng = np.random.default_rng(77)
    lw = rng.normal(size=7) * 2
    inc = rng.normal(size=7)
    assert np.array_equal(inc, g["small_inc"])
    for use_log in (0, 1):
        for cess in (0, 1):
            key = f"small_{'cess' if cess else 'ess'}_{use_log}"
            assert O.ref_weight_prospective(lw, inc, use_log, cess) == float(g[key])


def test_resample_m_ne_n_golden():
    """The C restatement's Resample(M, N) and cfrp_trans expansion against
    vSMC's (tests/golden/resample_mn.npz)."""
    import os

    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import MN_CASES

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "resample_mn.npz"))
    n = 0
    for M, N in MN_CASES:
        w = g[f"M{M}_N{N}_w"]
        for sch in range(6):
            for seed, skip in ((103, 0), (7, 5)):
                tag = f"M{M}_N{N}_s{sch}_{seed}_{skip}"
                rep, cf, words = O.resample(sch, w, seed, skip, M=M, N=N)
                assert np.array_equal(rep, g[tag + "_rep"]), tag
                assert np.array_equal(cf, g[tag + "_cf"]), tag
                assert words == int(g[tag + "_words"]), tag
                n += 1
    assert n == 12 * len(MN_CASES)
