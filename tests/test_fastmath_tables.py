"""The committed tables of the library's table-driven FP64 log and exp
(include/vsmc_b200/fastmath_tables.cuh) are what their generator writes,
and the generator's values are accurate double-doubles."""
import importlib.util
import os
from decimal import Decimal, getcontext

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GEN = os.path.join(ROOT, "include", "vsmc_b200", "gen_fastmath_tables.py")
TAB = os.path.join(ROOT, "include", "vsmc_b200", "fastmath_tables.cuh")


def load_gen():
    spec = importlib.util.spec_from_file_location("gen_fastmath_tables", GEN)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_tables_regenerate_identically(tmp_path):
    out = load_gen().main(str(tmp_path / "t.cuh"))
    with open(out) as a, open(TAB) as b:
        assert a.read() == b.read()


def parse(name):
    rows = []
    with open(TAB) as fh:
        inside = False
        for line in fh:
            if name in line and "[" in line:
                inside = True
                continue
            if inside:
                if line.startswith("};"):
                    break
                vals = line.strip().strip("{},").split(",")
                rows.append([float.fromhex(v.strip().strip("{}")) for v in vals])
    return rows


@pytest.mark.parametrize("name", ["kLogTab", "kExpTab"])
def test_table_values(name):
    getcontext().prec = 60
    rows = parse(name)
    if name == "kLogTab":
        assert len(rows) == 182
        for i, (c, hi, lo) in enumerate(rows):
            F = Decimal(181 + i) / 256
            assert abs(Decimal(c) * F - 1) < Decimal(2) ** -52
            exact = -Decimal(c).ln()
            assert abs(Decimal(hi) + Decimal(lo) - exact) <= abs(exact) * Decimal(2) ** -104
    else:
        assert len(rows) == 256
        for j, (hi, lo) in enumerate(rows):
            exact = Decimal(2) ** (Decimal(j) / 256)
            assert abs(Decimal(hi) + Decimal(lo) - exact) <= exact * Decimal(2) ** -104
