"""The move kernels compute the polar method's coordinate 2U - 1 of
libstdc++'s generate_canonical<double, 53> over two 32-bit words (the
reference's std::normal_distribution in example/pf/include/pf_smp.hpp:
207-238) as one fused multiply-add of the rounded 64-bit integer,
fma(d, 2^-63, -1), clamped to 1 - 2^-52.  This checks on the CPU, with exact
rational arithmetic, that the fused form equals the two-step form
(U = d * 2^-64 clamped below 1, then 2U - 1) for every kind of input: the
rounding edges of the 64-bit conversion, the clamp at 2^64 and random words.
"""
import random
from fractions import Fraction

import pytest

ONE_BELOW = float.fromhex("0x1.fffffffffffffp-1")   # largest double < 1
TWO_U_MAX = float.fromhex("0x1.ffffffffffffep-1")   # 2 * ONE_BELOW - 1


def two_step(x: int) -> float:
    d = float(x)  # round-half-even, like the device's __ull2double_rn
    u = d * 2.0 ** -64
    if u >= 1.0:
        u = ONE_BELOW
    return (2.0 * u) - 1.0


def fused(x: int) -> float:
    d = float(x)
    r = float(Fraction(d) * Fraction(1, 2 ** 63) - 1)  # one rounding
    return TWO_U_MAX if r >= 1.0 else r


EDGES = [0, 1, 2, 2 ** 32 - 1, 2 ** 32, 2 ** 53 - 1, 2 ** 53, 2 ** 53 + 1,
         2 ** 62 + 2 ** 9, 2 ** 62 + 2 ** 9 + 1, 2 ** 63 - 1, 2 ** 63,
         2 ** 63 + 2 ** 10, 2 ** 64 - 2 ** 11, 2 ** 64 - 2 ** 10 - 1,
         2 ** 64 - 2 ** 10, 2 ** 64 - 1]


@pytest.mark.parametrize("x", EDGES)
def test_edges(x):
    assert fused(x) == two_step(x)


def test_random_words():
    rng = random.Random(20)
    xs = [rng.getrandbits(64) for _ in range(20000)]
    xs += [rng.getrandbits(rng.randint(1, 64)) for _ in range(20000)]
    bad = [x for x in xs if fused(x) != two_step(x)]
    assert not bad, bad[:5]
