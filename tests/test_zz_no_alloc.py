"""The no-allocation resampler (vsmc_cuda_resample_noalloc) against the
workspace resampler (vsmc_cuda_resample).

Some callers cannot allocate device memory while they run: a process whose
HBM budget is fixed up front, a latency-critical loop where cudaMalloc would
synchronise the device, or a plugin whose host owns every allocation.  The
no-allocation entry point serves them from a static device array; here it
must give exactly the replication counts, copy_from indices and engine
words of the workspace entry point on the same inputs, for two calls in a
row (the second call runs on the scratch the first one left behind).  This
file is collected last so that a failure here does not stop the other
tests."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from vsmc_b200 import capi as C

    C.lib()
    return C


def _workspace_call(capi, sch, w_dev, N, rng):
    rep = torch.empty(N, dtype=torch.int32, device="cuda")
    cf = torch.empty(N, dtype=torch.int32, device="cuda")
    nb = capi.resample_workspace_size(N)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    words = capi.resample(sch, N, w_dev.data_ptr(), rng, rep.data_ptr(), cf.data_ptr(),
                          ws.data_ptr(), nb)
    return rep.cpu().numpy(), cf.cpu().numpy(), words


def _noalloc_call(capi, sch, w_dev, N, rng, with_cf=True):
    rep = torch.empty(N, dtype=torch.int32, device="cuda")
    cf = torch.empty(N, dtype=torch.int32, device="cuda") if with_cf else None
    words = capi.resample_noalloc(sch, N, w_dev.data_ptr(), rng, rep.data_ptr(),
                                  cf.data_ptr() if with_cf else None)
    return rep.cpu().numpy(), (cf.cpu().numpy() if with_cf else None), words


@pytest.mark.parametrize("sch", range(6))
def test_noalloc_matches_workspace_twice(capi, sch):
    rng_np = np.random.default_rng(100 + sch)
    for call, N in enumerate((capi.NOALLOC_MAX_N, 40000)):
        lw = rng_np.normal(size=N) * 2.0
        w = np.exp(lw - lw.max())
        w /= w.sum()
        w_dev = torch.from_numpy(w).cuda()
        a = capi.threefry_state(17, offset=3 + call)
        b = capi.threefry_state(17, offset=3 + call)
        ref = _workspace_call(capi, sch, w_dev, N, a)
        got = _noalloc_call(capi, sch, w_dev, N, b)
        assert np.array_equal(got[0], ref[0]), (sch, call)
        assert np.array_equal(got[1], ref[1]), (sch, call)
        assert got[2] == ref[2] and a.offset == b.offset


def test_noalloc_without_copy_from(capi):
    N = 5000
    w = np.random.default_rng(3).random(N)
    w /= w.sum()
    w_dev = torch.from_numpy(w).cuda()
    ref = _workspace_call(capi, 0, w_dev, N, capi.threefry_state(9))
    got = _noalloc_call(capi, 0, w_dev, N, capi.threefry_state(9), with_cf=False)
    assert np.array_equal(got[0], ref[0]) and got[2] == ref[2]


def test_noalloc_rejects_too_many_particles(capi):
    N = capi.NOALLOC_MAX_N + 1
    w_dev = torch.full((N,), 1.0 / N, dtype=torch.float64, device="cuda")
    rep = torch.empty(N, dtype=torch.int32, device="cuda")
    with pytest.raises(capi.VsmcCudaError) as e:
        capi.resample_noalloc(3, N, w_dev.data_ptr(), capi.threefry_state(1), rep.data_ptr(),
                              None)
    assert e.value.status == capi.EINVAL
    assert "static scratch limit" in str(e.value)
