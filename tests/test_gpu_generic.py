"""vsmc::Sampler<T> with moves the user compiles for the device
(include/vsmc_b200/smc.cuh), driven by tests/cpp/generic_main.cu:

- the constant-velocity Student-t filter written as vSMC user code (an
  InitializeCUDA and a MoveCUDA with __device__ initialize_state /
  move_state, a MonitorEvalCUDA for the position) prints vSMC's own
  summary table for the same filter (tests/golden/cv_summary_s*.tsv) byte
  for byte for all six schemes, with the log-evidence within 1e-9;
- the reference's example/paper/src/paper_pf.cpp model (its own sd, the
  default RngSet<Threefry4x64, Vector> and Stratified resampling) prints the
  table vSMC prints for it (tests/golden/paper_pf_summary.tsv, made by
  oracle/ref_paper_pf.cpp from the example's own classes)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
LIBDIR = os.path.join(ROOT, "vsmc_b200", "lib")

pytestmark = pytest.mark.gpu


def compile_generic(out_dir):
    exe = os.path.join(out_dir, "generic_main")
    cmd = [os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc"), "-std=c++17",
           "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false",
           "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "generic_main.cu"), "-o", exe,
           "-L", LIBDIR, "-lvsmc_cuda", "-Xlinker", f"-rpath={LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    return compile_generic(str(tmp_path_factory.mktemp("generic")))


def run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.split()


@pytest.mark.parametrize("sch", range(6))
def test_cv_user_model_matches_reference_table(golden, exe, tmp_path, sch):
    obs = tmp_path / "obs.bin"
    np.concatenate([golden["cv_obs_x"], golden["cv_obs_y"]]).tofile(obs)
    out = tmp_path / "est.tsv"
    logz = float(run(exe, "cv", 1000, 100, sch, obs, out)[0])
    with open(os.path.join(GOLDEN, f"cv_summary_s{sch}.tsv")) as f:
        want = f.read()
    assert out.read_text() == want
    ref = float(golden[f"cv_s{sch}_logz"])
    assert abs(logz - ref) <= 1e-9 * abs(ref)


def test_paper_pf_model_matches_reference_table(exe, tmp_path):
    g = np.load(os.path.join(GOLDEN, "paper_pf_obs.npz"))
    T, N = int(g["T"]), int(g["N"])
    obs = tmp_path / "obs.bin"
    np.concatenate([g["obs_x"], g["obs_y"]]).tofile(obs)
    out = tmp_path / "est.tsv"
    logz = float(run(exe, "paper", N, T, obs, out)[0])
    with open(os.path.join(GOLDEN, "paper_pf_summary.tsv")) as f:
        want = f.read()
    assert out.read_text() == want
    assert np.isfinite(logz)
