"""CPU checks of the C ABI: the library loads and exports every function
declared in include/vsmc_cuda.h (no device calls)."""
import os
import re

import pytest

from vsmc_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "vsmc_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vsmc_cuda_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    from vsmc_b200 import capi

    return capi.lib()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lib):
    from vsmc_b200 import capi

    assert lib.vsmc_cuda_abi_version() == 1
    for s in range(6):
        assert lib.vsmc_cuda_status_string(s).startswith(b"VSMC_CUDA_")
    assert capi.resample_workspace_size(0) == 0
    assert capi.resample_workspace_size(1 << 20) > 0


def test_config_validation_without_device(lib):
    from vsmc_b200 import capi

    c = capi.cv_config()
    assert c.threshold == 0.5 and c.seed == 101 and c.nu == 10.0
    assert capi.CVFilter.device_bytes(N=0, T_max=10) == 0          # N too small
    assert capi.CVFilter.device_bytes(N=1 << 20, T_max=100) > 40 * (1 << 20)
    assert capi.CVFilter.device_bytes(N=1 << 20, T_max=100, scheme=9) == 0
    mixed = capi.CVFilter.device_bytes(N=1 << 20, T_max=100, form=capi.MIXED)
    fp64 = capi.CVFilter.device_bytes(N=1 << 20, T_max=100)
    assert mixed < fp64


def test_sm100a_only_build():
    assert "arch=compute_100a,code=sm_100a" in " ".join(B.ARCH)


def test_product_simulator_matches_oracle(lib):
    """vsmc_cuda_cv_simulate (host code of the product) reproduces the
    oracle's observation series bit for bit."""
    import numpy as np

    from oracle import oracle as O
    from vsmc_b200 import capi

    for seed, stream in ((7, 0), (11, 3), (2**32 - 1, 2**31)):
        a = capi.cv_simulate(120, seed, stream_id=stream, want_truth=True)
        b = O.cv_simulate(120, seed, stream=stream, want_truth=True)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
