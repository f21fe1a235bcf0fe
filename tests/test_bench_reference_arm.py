"""bench.py's reference arm runs vSMC itself on the host (no GPU): its
JSON line carries the same metric and unit as the device arm, marks itself
"reference", and describes its CPU run."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ref_built():
    sys.path.insert(0, ROOT)
    from oracle import oracle as O

    return O.ref_available()


@pytest.mark.skipif(not _ref_built(), reason="oracle/_ref not built (run __graft_entry__.build())")
def test_reference_arm_line():
    out = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
         "--particles", "65536", "--steps", "3", "--warmup", "3"],
        capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "particle-steps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 3 and line["warmup"] == 3
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["particles"] == 65536
    # the device arm prints the same config object for the same workload
    sys.path.insert(0, ROOT)
    import bench

    assert line["config"] == bench.workload_config(
        65536, 7, "Multinomial", "fp64", 0.5, 1, line["config"]["resampled_steps"])
    assert line["config"]["workload"] == ("cv_student_t N=65536 T=7 Multinomial fp64 "
                                          "threshold 0.5 seed 101")
    assert line["state_std"]["kind"] == "reference" and line["state_std"]["value"] > 0


def test_bench_rejects_short_warmup():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--warmup", "2"],
                         capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert out.returncode != 0 and "--warmup must be >= 3" in out.stderr
