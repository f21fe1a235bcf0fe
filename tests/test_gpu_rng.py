"""Philox4x32-10 and Threefry4x64-20 word streams on the device against the
golden fixtures from the vSMC engines: bit-exact."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.gpu_util import empty

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from vsmc_b200 import capi as C

    C.lib()
    return C


@pytest.mark.parametrize("i", range(4))
def test_philox_golden(golden, capi, i):
    k, c = golden[f"philox_{i}_key"], golden[f"philox_{i}_ctr"]
    s = int(golden[f"philox_{i}_skip"])
    ref = golden[f"philox_{i}_words"]
    out = empty(ref.size, torch.int32)
    capi.philox4x32_words(tuple(int(x) for x in k), tuple(int(x) for x in c), s, ref.size,
                          out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)


@pytest.mark.parametrize("i", range(4))
def test_threefry_golden(golden, capi, i):
    k, c = golden[f"threefry_{i}_key"], golden[f"threefry_{i}_ctr"]
    s = int(golden[f"threefry_{i}_skip"])
    ref = golden[f"threefry_{i}_words"]
    out = empty(ref.size, torch.int64)
    capi.threefry4x64_words(tuple(int(x) for x in k), tuple(int(x) for x in c), s, ref.size,
                            out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), ref)


@pytest.mark.parametrize("skip", [0, 1, 2, 3, 5, 1 << 20])
def test_streams_large(capi, skip):
    """Millions of words, every skip alignment, against the C restatement."""
    n = (1 << 21) + 3
    key, ctr = (0xDEADBEEF, 12345), (0xFFFFFFF0, 0xFFFFFFFF, 7, 0)
    out = empty(n, torch.int32)
    capi.philox4x32_words(key, ctr, skip, n, out.data_ptr())
    k64, c64 = (1, 2, 3, 4), (2**64 - 3, 2**64 - 1, 0, 9)
    out64 = empty(n // 4, torch.int64)
    capi.threefry4x64_words(k64, c64, skip, n // 4, out64.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), O.philox_stream(key, ctr, n, skip))
    assert np.array_equal(out64.cpu().numpy().view(np.uint64),
                          O.threefry_stream(k64, c64, n // 4, skip))
