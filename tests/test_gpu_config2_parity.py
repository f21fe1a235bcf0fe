"""The device filter against vSMC itself at the benchmark's particle counts.

The reference is the unmodified vSMC Sampler (StateOMP, every host thread)
built by oracle/Makefile; it records each step's copy_from as
Particle::resample hands it to the value (core/particle.hpp:230-250).  The
device filter then follows the reference's ancestry step by step while it
still resamples on its own weights and its own engine position (the compare
mode of vsmc_cuda_cv_set_ancestry), so that both runs keep the same
particles and every step's resampling is compared on the same trajectory:

* the ESS history (which fixes every resampling decision), the log-evidence
  increments and the posterior-mean path agree to 1e-9 relative, and the
  decisions ESS < threshold * N are identical;
* the resample engine has drawn exactly the reference's words after every
  step;
* the number of replication counts and of copy_from entries that differ
  from the reference's is counted per step, and must be 0.  The device
  reproduces the reference's sequential sums bit for bit -- the cumulative
  weight `accw += w[i]` (resample/common.hpp:76-79), the normalising
  `asum` (core/weight_set.hpp:121) and the sorted sequence's `lmax_ +=`
  (rng/u01.hpp:185) -- so a count could differ only where the device's log
  or exp rounds differently from glibc's and a uniform lies within that
  rounding of a cumulative weight; none does in these runs.  (One differing
  count would shift every later surplus child in cfrp_trans's assignment,
  so copy_from differences would come in runs.)  The counts are printed
  (and written to $VSMC_PARITY_REPORT when set).
* Given the reference's own normalised weights and uniforms, the device
  resampler reproduces the reference's replication and copy_from of the
  same step exactly, for every scheme, at 2^24 particles.

The mixed form's log-evidence on the FP64 run's ancestry is checked at
2^24 particles over 100 steps (the benchmark's precision claim)."""
import json
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.gpu_util import dev, empty

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not O.ref_available(), reason="reference harness not built"),
]

RTOL = 1e-9
THRESHOLD = 1.1  # every step resamples
SEED = 101


@pytest.fixture(scope="module")
def capi():
    from vsmc_b200 import capi as C

    C.lib()
    return C


def report(key, value):
    path = os.environ.get("VSMC_PARITY_REPORT")
    if not path:
        return
    data = {}
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
    data[key] = value
    with open(path, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)


def rel_close(a, b, rtol=RTOL):
    a, b = np.asarray(a), np.asarray(b)
    return bool(np.all(np.abs(a - b) <= rtol * np.maximum(np.abs(b), 1e-300) + 1e-12))


def compare_run(capi, N, T, sch, obs_seed):
    ox, oy = O.cv_simulate(T, obs_seed=obs_seed)
    ref = O.ref_cv_filter_trace(N, T, sch, ox, oy, seed=SEED, threshold=THRESHOLD,
                                weights_step=0)
    assert np.all(ref["resampled"] == 1)
    rep = dev(ref["copy_from"])
    flags = dev(ref["resampled"].astype(np.int32))
    rec = torch.full((T, N), -1, dtype=torch.int32, device="cuda")
    words = []
    with capi.CVFilter(N, T, scheme=sch, seed=SEED, threshold=THRESHOLD) as f:
        f.set_ancestry(record_ptr=rec.data_ptr(), replay_ptr=rep.data_ptr(),
                       replay_flags_ptr=flags.data_ptr())
        f.set_observations_host(ox, oy)
        f.initialize()
        words.append(f.resample_words())
        for _ in range(T - 1):
            f.iterate(1)
            words.append(f.resample_words())
        h = f.history()
        h["logz"] = f.log_evidence()
    own = rec.cpu().numpy()
    mism = [int(np.count_nonzero(own[t] != ref["copy_from"][t])) for t in range(T)]
    rep_mism = [int(np.count_nonzero(np.bincount(own[t], minlength=N)
                                     != np.bincount(ref["copy_from"][t], minlength=N)))
                for t in range(T)]
    ref_words = [int(x) for x in ref["words_before"][1:]] + [ref["words_used"]]
    return ox, oy, ref, h, mism, rep_mism, words, ref_words


# (N, T, scheme, per-step bound on differing replication counts)
CASES = [((1 << 20), 8, s, 0) for s in range(6)] + [
    ((1 << 24), 6, 3, 0),
    ((1 << 24), 6, 2, 0),
    ((1 << 24), 6, 0, 0),
]


@pytest.mark.parametrize("N,T,sch,bound", CASES,
                         ids=[f"N{c[0]}-s{c[2]}" for c in CASES])
def test_filter_against_reference(capi, N, T, sch, bound):
    ox, oy, ref, h, mism, rep_mism, words, ref_words = compare_run(capi, N, T, sch,
                                                                   obs_seed=31)
    print(f"N={N} scheme {sch}: replication counts differing per step {rep_mism}, "
          f"copy_from entries {mism}; engine words {words} (reference {ref_words})")
    report(f"filter_N{N}_s{sch}", {"replication_mismatch_per_step": rep_mism,
                                   "copy_from_mismatch_per_step": mism, "words": words,
                                   "ref_words": ref_words})
    assert words == ref_words
    assert np.array_equal((h["ess"] < THRESHOLD * N).astype(np.int32), ref["resampled"])
    assert rel_close(h["ess"], ref["ess"])
    assert rel_close(h["logz_inc"], ref["logz_inc"])
    assert rel_close(h["mean_x"], ref["mean_x"]) and rel_close(h["mean_y"], ref["mean_y"])
    assert abs(h["logz"] - ref["logz"]) <= RTOL * abs(ref["logz"])
    assert max(rep_mism) <= bound


@pytest.mark.parametrize("sch", range(6))
def test_resampler_on_reference_weights(capi, sch):
    """Step 0 of the 2^24-particle run: the reference's normalised weights
    and engine position (and, for the log/exp sequences, the reference's
    uniforms through the pinned C restatement) into vsmc_cuda_resample;
    replication sums and engine words exact, copy_from compared with the
    reference's own row."""
    N, T = 1 << 24, 1
    ox, oy = O.cv_simulate(T, obs_seed=31)
    ref = O.ref_cv_filter_trace(N, T, sch, ox, oy, seed=SEED, threshold=THRESHOLD,
                                weights_step=0)
    w = ref["weights"]
    skip = int(ref["words_before"][0])
    uni = None
    if sch in (0, 1):
        _, ocf, owords, uni = O.resample(sch, w, SEED + 2, skip, want_uniforms=True)
        assert np.array_equal(ocf, ref["copy_from"][0])
    wd = dev(w)
    repd = empty(N, torch.int32)
    cfd = empty(N, torch.int32)
    nb = capi.resample_workspace_size(N)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    rng = capi.threefry_state(SEED + 2, offset=skip)
    up, nu = None, 0
    if uni is not None:
        ud = dev(uni)
        up, nu = ud.data_ptr(), uni.size
    words = capi.resample(sch, N, wd.data_ptr(), rng, repd.data_ptr(), cfd.data_ptr(),
                          ws.data_ptr(), nb, uniforms_ptr=up, n_uniforms=nu)
    cf = cfd.cpu().numpy()[:N]
    rep = repd.cpu().numpy()[:N]
    mism = int(np.count_nonzero(cf != ref["copy_from"][0]))
    rep_mism = int(np.count_nonzero(rep != np.bincount(ref["copy_from"][0], minlength=N)))
    print(f"resampler N={N} scheme {sch} on the reference's weights: "
          f"{rep_mism} replication counts and {mism} copy_from entries differ")
    report(f"resampler_N{N}_s{sch}", {"copy_from_mismatch": mism,
                                      "replication_mismatch": rep_mism})
    assert words == ref["words_used"] - skip
    assert rep.sum() == N
    assert rep_mism == 0 and mism == 0


def test_mixed_form_fixed_ancestry_benchmark_size(capi):
    """The mixed form (FP32 move and weights, FP64 scan and log-evidence) on
    the FP64 run's ancestry at the benchmark size: relative log-evidence
    error within 1e-6 over 100 steps (Multinomial, threshold 0.5)."""
    N, T = 1 << 24, 100
    ox, oy = capi.cv_simulate(T, 7)
    rec = torch.zeros((T, N), dtype=torch.int32, device="cuda")
    with capi.CVFilter(N, T, scheme=0) as f:
        f.set_ancestry(record_ptr=rec.data_ptr())
        f.set_observations_host(ox, oy)
        f.initialize()
        f.iterate(T - 1)
        h64 = f.history()
        z64 = f.log_evidence()
    flags = dev(h64["resampled"].astype(np.int32))
    with capi.CVFilter(N, T, scheme=0, form=capi.MIXED) as g:
        g.set_ancestry(replay_ptr=rec.data_ptr(), replay_flags_ptr=flags.data_ptr())
        g.set_observations_host(ox, oy)
        g.initialize()
        g.iterate(T - 1)
        z32 = g.log_evidence()
    err = abs(z64 - z32) / abs(z64)
    print(f"mixed form replay N={N}: logZ {z32:.12f} vs FP64 {z64:.12f}, rel err {err:.3e}")
    report("mixed_fixed_ancestry_N16M", {"rel_err": err, "logz64": z64, "logz32": z32})
    assert err <= 1e-6
