"""Regenerate the golden fixtures from the unmodified vSMC headers.

Run from the repository root where the vSMC include tree is available:

    make -C oracle && python tests/golden/make_golden.py

(`python tests/golden/make_golden.py summaries` rewrites only the summary
tables cv_summary_s*.tsv; `... gmm` only gmm.npz and gmm_summary.tsv, the
tempered SMC sampler of oracle/ref_gmm.cpp; `... paper` only
paper_pf_obs.npz and paper_pf_summary.tsv, the reference's example/paper
particle filter of oracle/ref_paper_pf.cpp; `... prospective` only
prospective.npz, WeightSet::ess / cess of incremental weights; `... mn`
only resample_mn.npz, resampling M weights into N != M children.)

Every array in golden.npz is produced by oracle/_ref/libvsmc_ref.so
(oracle/ref_harness.cpp over vSMC's own Sampler, WeightSet, Resample<...>,
internal::cfrp_trans, Philox4x32 and Threefry4x64).  The C restatement in
oracle/smc_oracle.c is then checked against these arrays by
tests/test_oracle.py, and the CUDA path against both by the gpu tests.
Observations are the workload's simulated series (oracle.cv_simulate: a
seeded Philox4x32-10 stream starting at state (0, 0, 1, 1)).
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")

PHILOX_CASES = [((0, 0), (0, 0, 0, 0), 0), ((102, 0), (0, 5, 7, 0), 3),
                ((0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF), 1),
                ((12345, 678), (0xFFFFFFFE, 0, 1 << 20, 9), 0)]
THREEFRY_CASES = [((0, 0, 0, 0), (0, 0, 0, 0), 0), ((103, 0, 0, 0), (0, 0, 0, 0), 5),
                  ((2**64 - 1,) * 4, (2**64 - 1,) * 4, 2),
                  ((1, 2, 3, 4), (2**64 - 2, 7, 0, 0), 0)]
NWORDS = 1027


def weight_cases(rng):
    """Weight vectors for the resample fixtures (name, w, N)."""
    cases = []
    for M in (1, 2, 3, 17, 1000, 4096):
        w = rng.random(M)
        cases.append((f"uniform_rand_{M}", w / w.sum(), M))
    M = 4096
    lw = rng.normal(size=M) * 3.0
    w = np.exp(lw - lw.max())
    cases.append(("lognormal_4096", w / w.sum(), M))
    w = np.zeros(M)
    w[1234] = 1.0
    cases.append(("degenerate_4096", w, M))
    w = np.full(M, 1.0 / M)
    cases.append(("equal_4096", w, M))
    k = rng.integers(0, 64, size=M).astype(np.float64)  # dyadic, exact partial sums
    k[0] += 1
    tot = 1 << int(np.ceil(np.log2(k.sum())))
    k[-1] += tot - k.sum()
    cases.append(("dyadic_4096", k / tot, M))
    w = rng.random(M)
    w[rng.random(M) < 0.5] = 0.0
    cases.append(("sparse_4096", w / w.sum(), M))
    w = rng.random(1000)
    cases.append(("N0_M1000", w / w.sum(), 0))
    return cases


def main():
    rng = np.random.default_rng(20240611)
    g = {}
    for i, (k, c, s) in enumerate(PHILOX_CASES):
        g[f"philox_{i}_key"] = np.array(k, np.uint32)
        g[f"philox_{i}_ctr"] = np.array(c, np.uint32)
        g[f"philox_{i}_skip"] = np.array(s, np.uint64)
        g[f"philox_{i}_words"] = O.philox_stream(k, c, NWORDS, s, use_ref=True)
    for i, (k, c, s) in enumerate(THREEFRY_CASES):
        g[f"threefry_{i}_key"] = np.array(k, np.uint64)
        g[f"threefry_{i}_ctr"] = np.array(c, np.uint64)
        g[f"threefry_{i}_skip"] = np.array(s, np.uint64)
        g[f"threefry_{i}_words"] = O.threefry_stream(k, c, NWORDS, s, use_ref=True)

    # WeightSet: set_log_weight then add_log_weight
    for i, (N, s_lw, s_inc) in enumerate([(1, 1.0, 1.0), (1000, 5.0, 3.0), (4096, 30.0, 50.0)]):
        lw = rng.normal(size=N) * s_lw
        inc = rng.normal(size=N) * s_inc
        ess, w, lwo = O.ref_weight_set(lw, inc)
        g[f"weight_{i}_lw"], g[f"weight_{i}_inc"] = lw, inc
        g[f"weight_{i}_ess"] = np.array(ess)
        g[f"weight_{i}_w"], g[f"weight_{i}_lwout"] = w, lwo

    names = []
    for name, w, N in weight_cases(rng):
        names.append(name)
        g[f"res_{name}_w"] = w
        g[f"res_{name}_N"] = np.array(N, np.int64)
        for sch in range(6):
            for seed, skip in ((103, 0), (7, 5)):
                rep, cf, words = O.ref_resample(sch, w, seed, skip, M=w.size, N=N)
                tag = f"res_{name}_s{sch}_{seed}_{skip}"
                g[tag + "_rep"] = rep.astype(np.int32)
                if N == w.size:
                    g[tag + "_cf"] = cf.astype(np.int32)
                g[tag + "_words"] = np.array(words, np.int64)
    g["res_names"] = np.array(names)

    # CV filter: N=1000, T=100 (the CPU-runnable configuration), all schemes
    T = 100
    ox, oy = O.cv_simulate(T, obs_seed=7)
    g["cv_obs_x"], g["cv_obs_y"] = ox, oy
    for sch in range(6):
        r = O.ref_cv_filter(1000, T, sch, ox, oy, seed=101, want_state=(sch == 0))
        for k in ("ess", "resampled", "logz_inc", "mean_x", "mean_y"):
            g[f"cv_s{sch}_{k}"] = r[k]
        g[f"cv_s{sch}_logz"] = np.array(r["logz"])
        g[f"cv_s{sch}_words"] = np.array(r["words_used"], np.int64)
        if sch == 0:
            g["cv_s0_state"] = r["state"]
            g["cv_s0_lw"] = r["lw"]
    # a second stream / seed at N=4096, T=30, systematic, threshold 0.8
    ox2, oy2 = O.cv_simulate(30, obs_seed=11, stream=3)
    g["cv2_obs_x"], g["cv2_obs_y"] = ox2, oy2
    r = O.ref_cv_filter(4096, 30, 3, ox2, oy2, seed=5, stream=3, threshold=0.8)
    for k in ("ess", "resampled", "logz_inc", "mean_x", "mean_y"):
        g[f"cv2_{k}"] = r[k]
    g["cv2_logz"] = np.array(r["logz"])
    np.savez_compressed(OUT, **g)
    print("wrote", OUT, os.path.getsize(OUT), "bytes,", len(g), "arrays")


def write_summaries():
    """cv_summary_s<scheme>.tsv: vSMC's `os << sampler` table for the N=1000,
    T=100 filter of golden.npz (same observations, seed 101)."""
    T = 100
    ox, oy = O.cv_simulate(T, obs_seed=7)
    here = os.path.dirname(os.path.abspath(__file__))
    for sch in range(6):
        text = O.ref_cv_summary(1000, T, sch, ox, oy, seed=101)
        with open(os.path.join(here, f"cv_summary_s{sch}.tsv"), "w") as f:
            f.write(text)


GMM_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gmm.npz")
# the tempered SMC fixture: N, iters, power, sweeps, sd, scheme, threshold, seed
GMM_RUN = dict(N=512, iters=20, power=4, sweeps=5, sd=0.1, scheme=3, threshold=0.5,
               seed=101)


def write_gmm():
    """gmm.npz: the tempered SMC sampler of example/gmm through vSMC
    (oracle/ref_gmm.cpp) on 1000 mixture points (seed 1)."""
    data = O.gmm_simulate(1000, 1)
    r = O.ref_gmm_smc(data, **GMM_RUN)
    g = {"data": data}
    for k in ("ess", "resampled", "zinc", "integrand", "grid", "accept", "params", "lw",
              "words"):
        g[k] = r[k]
    g["logz"] = np.array(r["logz"])
    g["path_logz"] = np.array(r["path_logz"])
    for k, v in GMM_RUN.items():
        g["run_" + k] = np.array(v)
    np.savez_compressed(GMM_OUT, **g)
    text = O.ref_gmm_summary(data, GMM_RUN["N"], GMM_RUN["iters"], GMM_RUN["sweeps"],
                             GMM_RUN["sd"], GMM_RUN["scheme"], GMM_RUN["threshold"],
                             GMM_RUN["seed"])
    with open(os.path.join(os.path.dirname(GMM_OUT), "gmm_summary.tsv"), "w") as f:
        f.write(text)


def write_prospective():
    """prospective.npz: WeightSet::ess(inc, use_log) and cess(inc, use_log)
    through vSMC for log-weights and increments of several shapes, with the
    normalised weights and log-weights WeightSet holds before the call."""
    rng = np.random.default_rng(77)
    g = {}
    cases = [("small", rng.normal(size=7) * 2, rng.normal(size=7)),
             ("wide", rng.normal(size=5000) * 5, rng.normal(size=5000) * 3),
             ("positive", rng.normal(size=4096), rng.uniform(0.1, 2.0, size=4096)),
             ("big", rng.normal(size=70001), rng.normal(size=70001) * 0.5)]
    for name, lw, inc in cases:
        _, w, lwn = O.ref_weight_set(lw)
        g[f"{name}_lw"] = lwn
        g[f"{name}_w"] = w
        g[f"{name}_inc"] = inc
        for use_log in (0, 1):
            for cess in (0, 1):
                g[f"{name}_{'cess' if cess else 'ess'}_{use_log}"] = np.array(
                    O.ref_weight_prospective(lw, inc, use_log, cess))
    np.savez_compressed(os.path.join(os.path.dirname(OUT), "prospective.npz"), **g)


MN_CASES = ((7, 12), (1000, 1731), (4096, 100), (3000, 3), (2, 9000))


def write_mn():
    """resample_mn.npz: Resample<Scheme>(M, N) and cfrp_trans(M, N) with
    M != N through vSMC (replication, copy_from, engine words) for random
    weights, every scheme and two engine positions."""
    rng = np.random.default_rng(5151)
    g = {}
    for M, N in MN_CASES:
        lw = rng.normal(size=M) * 2.0
        w = np.exp(lw - lw.max())
        w /= w.sum()
        g[f"M{M}_N{N}_w"] = w
        for sch in range(6):
            for seed, skip in ((103, 0), (7, 5)):
                rep, cf, words = O.ref_resample(sch, w, seed, skip, M=M, N=N)
                tag = f"M{M}_N{N}_s{sch}_{seed}_{skip}"
                g[tag + "_rep"] = rep
                g[tag + "_cf"] = cf
                g[tag + "_words"] = np.array(words)
    np.savez_compressed(os.path.join(os.path.dirname(OUT), "resample_mn.npz"), **g)


PAPER_RUN = dict(N=1000, T=100, seed=101, obs_seed=11)


def write_paper():
    """paper_pf_summary.tsv: `os << sampler` of the reference's
    example/paper/src/paper_pf.cpp model (its own classes, Stratified at
    ESS < N/2, Threefry4x64 engine per particle slot) on the workload's
    simulated series (obs seed 11), saved in paper_pf_obs.npz."""
    here = os.path.dirname(os.path.abspath(__file__))
    ox, oy = O.cv_simulate(PAPER_RUN["T"], obs_seed=PAPER_RUN["obs_seed"])
    text = O.ref_paper_pf_summary(PAPER_RUN["N"], PAPER_RUN["T"], ox, oy,
                                  seed=PAPER_RUN["seed"])
    np.savez_compressed(os.path.join(here, "paper_pf_obs.npz"), obs_x=ox, obs_y=oy,
                        **{k: np.array(v) for k, v in PAPER_RUN.items()})
    with open(os.path.join(here, "paper_pf_summary.tsv"), "w") as f:
        f.write(text)


if __name__ == "__main__":
    if sys.argv[1:] == ["gmm"]:
        write_gmm()
    elif sys.argv[1:] == ["paper"]:
        write_paper()
    elif sys.argv[1:] == ["prospective"]:
        write_prospective()
    elif sys.argv[1:] == ["mn"]:
        write_mn()
    else:
        if sys.argv[1:] != ["summaries"]:
            main()
            write_gmm()
            write_paper()
            write_prospective()
            write_mn()
        write_summaries()
