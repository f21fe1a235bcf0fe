"""The library's table-driven FP64 log and exp (include/vsmc_b200/fastmath.cuh)
against the C library's (glibc, through Python's math module, which the
reference's std::log / std::exp call) and CUDA's (torch.log / torch.exp on
the device): within one ulp of both everywhere, equal to glibc's on nearly
every input, and the special values right."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def capi():
    from vsmc_b200 import capi as C

    C.lib()
    return C


def dev_eval(capi, fn, x):
    xi = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
    out = torch.empty_like(xi)
    capi.math_eval(fn, xi.numel(), xi.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    return out.cpu().numpy(), xi


def ulps(a, b):
    """Distance in units in the last place between finite doubles."""
    def ordered(v):
        i = np.ascontiguousarray(v, dtype=np.float64).view(np.int64)
        return np.where(i < 0, -(i & np.int64(0x7FFFFFFFFFFFFFFF)), i)

    return np.abs(ordered(a) - ordered(b))


def log_inputs(rng, n):
    parts = [
        np.exp(rng.uniform(-700, 700, n)),            # the whole range
        1.0 + rng.uniform(-1e-3, 1e-3, n // 4),        # near 1
        rng.uniform(0.0, 1.0, n // 4),                 # r2 of the polar method
        1.0 + rng.uniform(0.0, 50.0, n // 4),          # (1 + a)(1 + b)
        np.ldexp(rng.uniform(1.0, 2.0, n // 16), rng.integers(-1074, -1022, n // 16)),
    ]
    return np.concatenate(parts)


def exp_inputs(rng, n):
    parts = [
        rng.uniform(-745.0, 709.7, n),
        rng.uniform(-40.0, 0.0, n // 2),              # weights exp(lw - M)
        rng.uniform(-1e-6, 1e-6, n // 8),
        rng.uniform(-745.1, -708.0, n // 8),          # subnormal results
    ]
    return np.concatenate(parts)


@pytest.mark.parametrize("fn", [0, 1])
def test_against_glibc_and_cuda(capi, fn):
    rng = np.random.default_rng(11 + fn)
    x = log_inputs(rng, 1 << 17) if fn == 0 else exp_inputs(rng, 1 << 17)
    got, xd = dev_eval(capi, fn, x)
    cuda = (torch.log(xd) if fn == 0 else torch.exp(xd)).cpu().numpy()
    f = math.log if fn == 0 else math.exp
    ref = np.array([f(v) for v in x.tolist()])
    fin = np.isfinite(ref) & (ref != 0.0)
    d_glibc = ulps(got[fin], ref[fin])
    d_cuda = ulps(got[fin], cuda[fin])
    # equality is counted on normal results (a subnormal exp is rounded
    # twice: once to 53 bits, once into the subnormal range)
    normal = np.abs(ref[fin]) >= 2.0 ** -1022
    same = float(np.mean(d_glibc[normal] == 0))
    print(f"{'log' if fn == 0 else 'exp'}: max ulp vs glibc {d_glibc.max()}, vs CUDA "
          f"{d_cuda.max()}; equal to glibc {100 * same:.4f}%, CUDA equal to glibc "
          f"{100 * float(np.mean(ulps(cuda[fin], ref[fin]) == 0)):.4f}%")
    assert d_glibc.max() <= 1 and d_cuda.max() <= 1
    assert same >= 0.999
    # zero results (exp underflow) agree too
    assert np.array_equal(got[ref == 0.0], ref[ref == 0.0])


def test_special_values(capi):
    x = np.array([0.0, -0.0, -1.0, np.inf, -np.inf, np.nan, 1.0, 5e-324, 2.0 ** -1022])
    got, _ = dev_eval(capi, 0, x)
    assert got[0] == -np.inf and got[1] == -np.inf
    assert np.isnan(got[2]) and got[3] == np.inf and np.isnan(got[4]) and np.isnan(got[5])
    assert got[6] == 0.0
    assert got[7] == math.log(5e-324) and got[8] == math.log(2.0 ** -1022)
    x = np.array([0.0, -0.0, 710.0, -746.0, np.inf, -np.inf, np.nan, 709.78, -745.13,
                  1e-300, -708.0, 708.0])
    got, _ = dev_eval(capi, 1, x)
    assert got[0] == 1.0 and got[1] == 1.0
    assert got[2] == np.inf and got[3] == 0.0 and got[4] == np.inf and got[5] == 0.0
    assert np.isnan(got[6])
    for i in (7, 8, 9, 10, 11):
        assert abs(got[i] - math.exp(x[i])) <= abs(math.exp(x[i])) * 2.3e-16 or \
            got[i] == math.exp(x[i])
