"""Device resampling (all six schemes) against the vSMC reference.

Given identical normalised weights and identical uniforms, replication,
copy_from and the number of resample-engine words drawn are bit-exact
(Stratified / Systematic draw their uniforms on the device from the same
Threefry4x64 words; Multinomial / Residual go through log and exp, so the
bit-exact comparison feeds the reference's U01 sequence in parity mode and the
device-drawn sequence is checked separately)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.gpu_util import dev, empty

pytestmark = pytest.mark.gpu

LOG_EXP_SCHEMES = (0, 1)  # Multinomial, Residual: sorted sequence via log/exp


@pytest.fixture(scope="module")
def capi():
    from vsmc_b200 import capi as C

    C.lib()
    return C


def gpu_resample(capi, scheme, w, seed, skip, uniforms=None):
    N = w.size
    wd = dev(w)
    rep = empty(N, torch.int32)
    cf = empty(N, torch.int32)
    nb = capi.resample_workspace_size(N)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    rng = capi.threefry_state(seed, offset=skip)
    up, nu = None, 0
    if uniforms is not None and uniforms.size > 0:
        ud = dev(uniforms)
        up, nu = ud.data_ptr(), uniforms.size
    words = capi.resample(scheme, N, wd.data_ptr(), rng, rep.data_ptr(), cf.data_ptr(),
                          ws.data_ptr(), nb, uniforms_ptr=up, n_uniforms=nu)
    return rep.cpu().numpy()[:N], cf.cpu().numpy()[:N], words


def cases(golden):
    for name in golden["res_names"]:
        name = str(name)
        w = golden[f"res_{name}_w"]
        if int(golden[f"res_{name}_N"]) != w.size:
            continue  # the device resampler is Particle::resample's M == N form
        for sch in range(6):
            for seed, skip in ((103, 0), (7, 5)):
                yield name, w, sch, seed, skip


def test_golden_bit_exact(golden, capi):
    n = 0
    for name, w, sch, seed, skip in cases(golden):
        tag = f"res_{name}_s{sch}_{seed}_{skip}"
        uni = None
        if sch in LOG_EXP_SCHEMES:
            _, _, _, uni = O.resample(sch, w, seed, skip, want_uniforms=True)
        rep, cf, words = gpu_resample(capi, sch, w, seed, skip, uni)
        assert np.array_equal(rep, golden[tag + "_rep"]), tag
        assert np.array_equal(cf, golden[tag + "_cf"]), tag
        assert words == int(golden[tag + "_words"]), tag
        n += 1
    assert n >= 100


@pytest.mark.parametrize("sch", LOG_EXP_SCHEMES)
def test_device_sorted_sequence(golden, capi, sch):
    """Device-drawn sorted U01 sequence (log/exp on the GPU): same words
    drawn; replication equal except where a uniform lies within a few ulps
    of a cumulative weight (none expected at these sizes)."""
    for name, w, s, seed, skip in cases(golden):
        if s != sch:
            continue
        tag = f"res_{name}_s{sch}_{seed}_{skip}"
        rep, cf, words = gpu_resample(capi, sch, w, seed, skip)
        assert words == int(golden[tag + "_words"]), tag
        assert np.abs(rep - golden[tag + "_rep"]).sum() <= 2, tag


@pytest.mark.parametrize("N", [1, 2, 3, 2047, 2048, 2049, 1 << 16, (1 << 20) + 37])
@pytest.mark.parametrize("sch", range(6))
def test_sizes_against_oracle(capi, N, sch):
    rng = np.random.default_rng(N * 7 + sch)
    lw = rng.normal(size=N) * 2.0
    w = np.exp(lw - lw.max())
    w /= w.sum()
    ref_rep, ref_cf, ref_words, uni = O.resample(sch, w, 103, 3, want_uniforms=True)
    rep, cf, words = gpu_resample(capi, sch, w, 103, 3,
                                  uni if sch in LOG_EXP_SCHEMES else None)
    assert words == ref_words
    assert np.array_equal(rep, ref_rep)
    assert np.array_equal(cf, ref_cf)


@pytest.mark.parametrize("sch", range(6))
def test_invariants_and_determinism(capi, sch):
    """Size-independent properties at 2^22: sum rep = N, survivors keep
    their slot, sources are survivors, bincount(copy_from) = rep, and two
    runs are bitwise identical."""
    N = 1 << 22
    rng = np.random.default_rng(sch)
    lw = rng.normal(size=N) * 3.0
    w = np.exp(lw - lw.max())
    w /= w.sum()
    a = gpu_resample(capi, sch, w, 11, 0)
    b = gpu_resample(capi, sch, w, 11, 0)
    rep, cf, words = a
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    assert rep.sum() == N and rep.min() >= 0
    idx = np.arange(N)
    assert np.array_equal(cf[rep > 0], idx[rep > 0])
    assert np.all(rep[cf] > 0)
    assert np.array_equal(np.bincount(cf, minlength=N), rep)


@pytest.mark.parametrize("stride", [3001, 40000])
@pytest.mark.parametrize("sch", [0, 3, 4])
def test_sparse_parents_against_oracle(capi, stride, sch):
    """Weight only on every stride-th particle (and the last one): each
    parent has thousands of children, so the empty slots of one tile take
    their parents from other tiles, up to tens of tiles away."""
    N = (1 << 17) + 5
    rng = np.random.default_rng(stride + sch)
    w = np.zeros(N)
    w[::stride] = rng.uniform(0.5, 1.5, size=len(w[::stride]))
    w[-1] = 1.0
    w /= w.sum()
    ref_rep, ref_cf, ref_words, uni = O.resample(sch, w, 29, 1, want_uniforms=True)
    rep, cf, words = gpu_resample(capi, sch, w, 29, 1,
                                  uni if sch in LOG_EXP_SCHEMES else None)
    assert words == ref_words
    assert np.array_equal(rep, ref_rep)
    assert np.array_equal(cf, ref_cf)


@pytest.mark.parametrize("sch", [0, 3, 4])
def test_invariants_near_maximum_size(capi, sch):
    """At 2^27 + 5 particles (8x the benchmark; the 32-bit counts and
    indices of the inversion and cfrp fill at scale): sum rep = N, survivors
    keep their slot, every copy_from source is a survivor, bincount of
    copy_from equals rep, the engine advanced, and a second call repeats the
    first bit for bit."""
    N = (1 << 27) + 5
    rng = np.random.default_rng(sch + 40)
    w = rng.gamma(0.5, size=N)
    w /= w.sum()
    a = gpu_resample(capi, sch, w, 17, 0)
    b = gpu_resample(capi, sch, w, 17, 0)
    rep, cf, words = a
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    assert words > 0
    assert rep.sum() == N and rep.min() >= 0
    keep = rep > 0
    assert np.array_equal(cf[keep], np.nonzero(keep)[0])
    assert np.all(keep[cf])
    assert np.array_equal(np.bincount(cf, minlength=N), rep)


def test_degenerate_and_equal_weights(capi):
    N = 1 << 16
    w = np.zeros(N)
    w[N // 3] = 1.0
    for sch in range(6):
        rep, cf, _ = gpu_resample(capi, sch, w, 5, 0)
        assert rep[N // 3] == N and np.all(cf == N // 3)
    w = np.full(N, 1.0 / N)
    for sch in (2, 3, 5):  # every slot keeps exactly one child
        rep, cf, _ = gpu_resample(capi, sch, w, 5, 0)
        assert np.all(rep == 1) and np.array_equal(cf, np.arange(N))


@pytest.mark.parametrize("i", range(3))
def test_weight_add_log(golden, capi, i):
    lw = golden[f"weight_{i}_lw"].copy()
    inc = golden[f"weight_{i}_inc"]
    N = lw.size
    lwd, incd, wd = dev(lw), dev(inc), empty(N, torch.float64)
    capi.weight_add_log(N, lwd.data_ptr())                         # set_log_weight
    ess = capi.weight_add_log(N, lwd.data_ptr(), wd.data_ptr(), incd.data_ptr())
    assert np.array_equal(lwd.cpu().numpy(), golden[f"weight_{i}_lwout"])
    np.testing.assert_allclose(wd.cpu().numpy()[:N], golden[f"weight_{i}_w"], rtol=1e-13,
                               atol=1e-300)
    assert abs(ess - float(golden[f"weight_{i}_ess"])) <= 1e-12 * float(golden[f"weight_{i}_ess"])


def test_weight_add_log_degenerate(capi):
    lw = dev(np.full(1000, -np.inf))
    with pytest.raises(capi.VsmcCudaError) as e:
        capi.weight_add_log(1000, lw.data_ptr())
    assert e.value.status == capi.EDEGENERATE


def test_copy_f64(capi):
    N = 5000
    src = np.random.default_rng(0).normal(size=(3, N))
    cf = np.random.default_rng(1).integers(0, N, size=N).astype(np.int32)
    s, d, c = dev(src), empty(3 * N, torch.float64), dev(cf)
    capi.copy_f64(N, 3, s.data_ptr(), d.data_ptr(), c.data_ptr())
    assert np.array_equal(d.cpu().numpy().reshape(3, N), src[:, cf])


def test_bad_arguments(capi):
    with pytest.raises(capi.VsmcCudaError) as e:
        capi.resample(7, 10, 0, capi.threefry_state(1), None, None, None, 0)
    assert e.value.status == capi.EINVAL


def gpu_resample_mn(capi, scheme, w, N, seed, skip, uniforms=None):
    M = w.size
    wd = dev(w)
    rep = empty(M, torch.int32)
    cf = empty(max(N, 1), torch.int32)
    nb = capi.resample_mn_workspace_size(M, N)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    rng = capi.threefry_state(seed, offset=skip)
    up, nu = None, 0
    if uniforms is not None and uniforms.size > 0:
        ud = dev(uniforms)
        up, nu = ud.data_ptr(), uniforms.size
    words = capi.resample_mn(scheme, M, N, wd.data_ptr(), rng, rep.data_ptr(),
                             cf.data_ptr(), ws.data_ptr(), nb, uniforms_ptr=up, n_uniforms=nu)
    return rep.cpu().numpy()[:M], cf.cpu().numpy()[:N], words


def test_golden_m_ne_n_bit_exact(golden, capi):
    """Resample(M, N) with M != N and cfrp_trans's expansion branch
    (resample/common.hpp:110-117) on the golden cases whose N differs from
    the number of weights."""
    n = 0
    for name in golden["res_names"]:
        name = str(name)
        w = golden[f"res_{name}_w"]
        N = int(golden[f"res_{name}_N"])
        if N == w.size or w.size == 0:
            continue
        for sch in range(6):
            for seed, skip in ((103, 0), (7, 5)):
                tag = f"res_{name}_s{sch}_{seed}_{skip}"
                uni = None
                if sch in LOG_EXP_SCHEMES:
                    _, _, _, uni = O.resample(sch, w, seed, skip, M=w.size, N=N,
                                              want_uniforms=True)
                rep, cf, words = gpu_resample_mn(capi, sch, w, N, seed, skip, uni)
                assert np.array_equal(rep, golden[tag + "_rep"]), tag
                assert cf.size == N
                assert words == int(golden[tag + "_words"]), tag
                n += 1
    assert n >= 12


def test_m_ne_n_golden_bit_exact(capi):
    """Resample(M, N) + cfrp_trans expansion against vSMC's own results
    (tests/golden/resample_mn.npz)."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import MN_CASES

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "resample_mn.npz"))
    for M, N in MN_CASES:
        w = g[f"M{M}_N{N}_w"]
        for sch in range(6):
            for seed, skip in ((103, 0), (7, 5)):
                tag = f"M{M}_N{N}_s{sch}_{seed}_{skip}"
                uni = None
                if sch in LOG_EXP_SCHEMES:
                    _, _, _, uni = O.resample(sch, w, seed, skip, M=M, N=N,
                                              want_uniforms=True)
                rep, cf, words = gpu_resample_mn(capi, sch, w, N, seed, skip, uni)
                assert np.array_equal(rep, g[tag + "_rep"]), tag
                assert np.array_equal(cf, g[tag + "_cf"]), tag
                assert words == int(g[tag + "_words"]), tag


@pytest.mark.parametrize("M,N", [(3000, (1 << 17) + 11), ((1 << 16) + 3, 5000),
                                 (1, 777), (4097, 2)])
@pytest.mark.parametrize("sch", range(6))
def test_m_ne_n_against_oracle(capi, M, N, sch):
    rng = np.random.default_rng(M + 13 * sch)
    lw = rng.normal(size=M) * 2.0
    w = np.exp(lw - lw.max())
    w /= w.sum()
    ref_rep, ref_cf, ref_words, uni = O.resample(sch, w, 19, 2, M=M, N=N,
                                                 want_uniforms=True)
    rep, cf, words = gpu_resample_mn(capi, sch, w, N, 19, 2,
                                     uni if sch in LOG_EXP_SCHEMES else None)
    assert words == ref_words
    assert rep.sum() == N
    assert np.array_equal(rep, ref_rep)
    assert np.array_equal(cf, ref_cf)


def test_m_ne_n_zero_children(capi):
    w = np.full(10, 0.1)
    for sch in range(6):
        rep, cf, words = gpu_resample_mn(capi, sch, w, 0, 5, 0)
        assert np.all(rep == 0)
        assert words == (1 if sch in (3, 5) else 0)


def test_prospective_ess_cess(capi):
    """WeightSet::ess(inc, use_log) and cess(inc, use_log) against vSMC's
    values (tests/golden/prospective.npz), relative 1e-10."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "prospective.npz"))
    for name in ("small", "wide", "positive", "big"):
        lw, w, inc = dev(g[f"{name}_lw"]), dev(g[f"{name}_w"]), dev(g[f"{name}_inc"])
        N = g[f"{name}_lw"].size
        for use_log in (0, 1):
            ess = capi.weight_ess(N, lw.data_ptr(), w.data_ptr(), inc.data_ptr(), use_log)
            cess = capi.weight_cess(N, w.data_ptr(), inc.data_ptr(), use_log)
            want_e = float(g[f"{name}_ess_{use_log}"])
            want_c = float(g[f"{name}_cess_{use_log}"])
            assert abs(ess - want_e) <= 1e-10 * abs(want_e), (name, use_log, ess, want_e)
            assert abs(cess - want_c) <= 1e-10 * abs(want_c), (name, use_log, cess, want_c)


@pytest.mark.parametrize("sch", range(6))
def test_benchmark_size_bit_exact(capi, sch):
    """At 2^24 particles (the benchmark size) with random weights, the device
    resampler equals the oracle's restatement of the reference (sequential
    `accw += w[i]`, resample/common.hpp:76-79) exactly: replication,
    copy_from and engine words."""
    N = 1 << 24
    rng = np.random.default_rng(2024 + sch)
    lw = rng.normal(size=N) * 2.0
    w = np.exp(lw - lw.max())
    w /= w.sum()
    ref_rep, ref_cf, ref_words, uni = O.resample(sch, w, 103, 7, want_uniforms=True)
    rep, cf, words = gpu_resample(capi, sch, w, 103, 7,
                                  uni if sch in LOG_EXP_SCHEMES else None)
    assert words == ref_words
    assert np.array_equal(rep, ref_rep)
    assert np.array_equal(cf, ref_cf)


@pytest.mark.parametrize("sch", [0, 2, 3])
def test_tie_heavy_weights_bit_exact(capi, sch):
    """Weights whose every addition to the running sum is a rounding tie
    (0.5 followed by 2^-54 steps: the sequential sum stays at 0.5 by
    round-half-even while the exact sum grows), so every tile holds more
    special elements than it keeps and is summed element by element; with
    runs of ordinary weights between them.  Equal to the oracle bit for
    bit."""
    N = (1 << 18) + 123
    rng = np.random.default_rng(sch)
    w = rng.uniform(0.5, 1.5, size=N) * (0.5 / N)
    w[: N // 3] = 2.0 ** -54
    w[0] = 0.5
    w[N // 3: N // 3 + 5000] = 2.0 ** -60
    ref_rep, ref_cf, ref_words, uni = O.resample(sch, w, 77, 0, want_uniforms=True)
    rep, cf, words = gpu_resample(capi, sch, w, 77, 0,
                                  uni if sch in LOG_EXP_SCHEMES else None)
    assert words == ref_words
    assert np.array_equal(rep, ref_rep)
    assert np.array_equal(cf, ref_cf)


@pytest.mark.parametrize("sch", LOG_EXP_SCHEMES)
def test_benchmark_size_device_sequence(capi, sch):
    """The sorted U01 sequence drawn on the device at 2^24: its lmax is the
    reference's sequential sum exactly (exact scan of the negated terms), so
    replication can differ from the oracle's only where the device's log or
    exp rounds differently from glibc's and a uniform lies within that
    rounding of a cumulative weight."""
    N = 1 << 24
    rng = np.random.default_rng(4242 + sch)
    lw = rng.normal(size=N) * 2.0
    w = np.exp(lw - lw.max())
    w /= w.sum()
    ref_rep, ref_cf, ref_words, _ = O.resample(sch, w, 103, 7, want_uniforms=True)
    rep, cf, words = gpu_resample(capi, sch, w, 103, 7)
    mism = int(np.count_nonzero(rep != ref_rep))
    print(f"scheme {sch} N={N}: {mism} replication counts differ from the oracle")
    assert words == ref_words
    assert rep.sum() == N
    assert mism <= 16
