"""Writes fastmath_tables.cuh: the tables of the table-driven FP64 log and
exp in fastmath.cuh (P. T. P. Tang, "Table-driven implementation of the
exponential function in IEEE floating-point arithmetic", ACM TOMS 15(2),
1989, and "Table-driven implementation of the logarithm function in IEEE
floating-point arithmetic", ACM TOMS 16(4), 1990).

Every value is computed with Python's decimal module at 60 digits and
split into a double-double (hi + lo, each rounded to nearest).

    python include/vsmc_b200/gen_fastmath_tables.py [output path]
"""
import os
import struct
import sys
from decimal import Decimal, getcontext

getcontext().prec = 60

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "fastmath_tables.cuh")

LOG_SPACING = 256          # log: F_j = j / 256 for m' in [sqrt(1/2), sqrt(2))
LOG_J0 = 181               # round(256 sqrt(1/2))
LOG_J1 = 362               # round(256 sqrt(2))
EXP_N = 256                # exp: 2^(j / 256), j = 0..255


def split(v: Decimal):
    hi = float(v)
    lo = float(v - Decimal(hi))
    return hi, lo


def trim(x: float, bits: int) -> float:
    """x with its mantissa cut to `bits` significant bits (toward zero)."""
    (u,) = struct.unpack("<Q", struct.pack("<d", x))
    drop = 53 - bits
    u &= ~((1 << drop) - 1)
    return struct.unpack("<d", struct.pack("<Q", u))[0]


def lit(x: float) -> str:
    return float.hex(x)


def main(out=OUT):
    ln2 = Decimal(2).ln()
    lines = [
        "// fastmath_tables.cuh -- written by gen_fastmath_tables.py; do not edit.",
        "#pragma once",
        "",
        "namespace vsmc_b200 {",
        "namespace fm {",
        "",
    ]
    # ln 2 with 42 significant bits, so that k * LN2_HI is exact for
    # |k| <= 2^11
    ln2_hi = trim(float(ln2), 42)
    ln2_lo = float(ln2 - Decimal(ln2_hi))
    lines += [f"constexpr double kLn2Hi = {lit(ln2_hi)};",
              f"constexpr double kLn2Lo = {lit(ln2_lo)};", ""]
    # log: c_j = 1 / F_j (rounded), L_j = -log(c_j) as hi + lo
    n_log = LOG_J1 - LOG_J0 + 1
    rows = []
    for j in range(LOG_J0, LOG_J1 + 1):
        F = Decimal(j) / LOG_SPACING
        c = float(Decimal(1) / F)
        L = -Decimal(c).ln()
        hi, lo = split(L)
        rows.append((c, hi, lo))
    lines.append(f"constexpr int kLogJ0 = {LOG_J0};")
    lines.append(f"constexpr int kLogN = {n_log};")
    lines.append("// {1 / F_j, -log(c_j) hi, -log(c_j) lo}, F_j = (kLogJ0 + i) / 256")
    lines.append(f"static __device__ const double kLogTab[{n_log}][3] = {{")
    for c, hi, lo in rows:
        lines.append(f"    {{{lit(c)}, {lit(hi)}, {lit(lo)}}},")
    lines.append("};")
    lines.append("")
    # exp: ln2 / 256 with 35 significant bits (n * hi exact for |n| < 2^18)
    c = ln2 / EXP_N
    c_hi = trim(float(c), 35)
    c_lo = float(c - Decimal(c_hi))
    inv = float(EXP_N / ln2)
    lines += [f"constexpr int kExpN = {EXP_N};",
              f"constexpr double kExpInv = {lit(inv)}; // 256 / ln 2",
              f"constexpr double kExpCHi = {lit(c_hi)}; // ln 2 / 256, hi",
              f"constexpr double kExpCLo = {lit(c_lo)};", ""]
    lines.append("// {2^(j/256) hi, lo}")
    lines.append(f"static __device__ const double kExpTab[{EXP_N}][2] = {{")
    for j in range(EXP_N):
        v = Decimal(2) ** (Decimal(j) / EXP_N)
        hi, lo = split(v)
        lines.append(f"    {{{lit(hi)}, {lit(lo)}}},")
    lines.append("};")
    lines += ["", "} // namespace fm", "} // namespace vsmc_b200", ""]
    with open(out, "w") as fh:
        fh.write("\n".join(lines))
    return out


if __name__ == "__main__":
    print(main(*sys.argv[1:2]))
