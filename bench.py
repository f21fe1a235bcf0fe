#!/usr/bin/env python3
"""SMC step throughput on B200: the constant-velocity Student-t bootstrap
filter at N = 2^24 particles, Multinomial resampling, FP64, one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--particles P] [--scheme NAME] [--form fp64|mixed]

A "step" is one SMC iteration over all particles: move + log-likelihood +
log-weight update, normalisation / ESS / log-evidence, resampling when
ESS < N/2, posterior-mean monitor (Sampler::iterate(1)).  The run is
initialize + W untimed steps + K timed steps over a simulated observation
series of length 1 + W + K.

value    particle-steps/s summed over GPUs, device-timed with CUDA events on the
         filter's stream, max over ranks, inputs resident in HBM.
e2e      the same metric through the C ABI with the observation of every step
         copied from pinned host memory and the step's ESS / log-evidence
         increment / resampled flag read back before the next step.
roofline the move kernel (dominant): algorithmic bytes per launch (80 B per
         particle FP64, 40 B mixed) over its CUDA-event duration, against the
         measured HBM copy bandwidth.
cpu_baseline  the vSMC reference (StateOMP over the unmodified headers, all
         host threads) on a bounded sample of the same workload.

N > 1 GPUs: independent filter replicas, one per rank (different counter
streams), no collective on the data path ("replicas only").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = ("particle-steps/s at N=2^24 + batched filters/s, p50/p99 latency, "
          "FP32 vs FP64 form")
UNIT = "particle-steps/s"
SCHEMES = ("Multinomial", "Residual", "Stratified", "Systematic",
           "ResidualStratified", "ResidualSystematic")
OBS_SEED = 7
# algorithmic bytes per particle-step (move) and per resampled particle
B_MOVE = {"fp64": 80, "mixed": 40}
B_RES = {"fp64": 76, "mixed": 40}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(form, N):
    """DRAM bytes per move launch from the committed ncu summary, scaled to N."""
    p = os.path.join(ROOT, "profiles", "move_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d[form]
        return float(e["dram_bytes_per_launch"]) * N / float(e["particles"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def rank_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def cpu_reference(N, scheme, warmup, steps, sample_steps=None, backend=0,
                  threshold=0.5):
    """The vSMC reference (oracle/_ref harness; backend 0 StateOMP, 1
    StateSTD; all host threads) on the same filter.  Returns (particle-steps/s
    over the timed steps, info)."""
    from oracle import oracle as O

    T = 1 + warmup + steps if sample_steps is None else 1 + sample_steps
    first = 1 + (warmup if sample_steps is None else 0)
    ox, oy = O.cv_simulate(T, obs_seed=OBS_SEED)
    resampled = None
    if O.ref_available():
        r = O.ref_cv_filter(N, T, scheme, ox, oy, seed=101, backend=backend,
                            threshold=threshold)
        timed = r["step_seconds"][first:]
        resampled = int(r["resampled"][first:].sum())
        kind, cores = "reference", (O.ref_max_threads() if backend == 0
                                    else os.cpu_count())
    else:
        t0 = time.perf_counter()
        O.cv_filter(N, T, scheme, ox, oy, seed=101, threshold=threshold)
        timed = [time.perf_counter() - t0]
        kind, cores = "port", 1
    n_steps = len(timed) if kind == "reference" else T
    return N * n_steps / float(sum(timed)), {"kind": kind, "cores": cores,
                                             "steps": n_steps, "resampled": resampled}


def workload_config(N, T, scheme, form, threshold, world, resampled):
    """The `config` object both arms print for the same workload."""
    return {"workload": f"cv_student_t N={N} T={T} {scheme} {form} "
                        f"threshold {threshold} seed 101",
            "particles": N, "scheme": scheme, "form": form,
            "resampled_steps": resampled,
            "l2": "inputs larger than L2 (state 512 MiB FP64 / 256 MiB mixed)",
            "parallelism": "replicas" if world > 1 else "single"}


def forms_compare(capi, N, sch, K, W, ox, oy, sp, fp64_step_ms):
    """Mixed form (float move / weights, double scan and log-evidence) against
    the FP64 form on the same inputs: device step time, and the relative
    log-evidence error on the FP64 run's ancestry (the mixed run replays the
    FP64 run's resampling decisions and copy_from vectors)."""
    import torch

    T = 1 + W + K
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.ExternalStream(sp)
    with capi.CVFilter(N, T, scheme=sch, form=capi.MIXED, seed=101, stream=sp) as m:
        m.set_observations_host(ox, oy)
        m.initialize()
        m.iterate(W)
        m.synchronize()
        e0.record(stream)
        m.iterate(K)
        e1.record(stream)
        m.synchronize()
        torch.cuda.synchronize()
        mixed_ms = e0.elapsed_time(e1) / K
        m.initialize()
        m.iterate(W)
        m.set_timing(True)
        m.iterate(K)
        mv_ms, st_ms, n, _ = m.timing()
    # fixed ancestry: record the FP64 run, replay it in the mixed form
    rec = torch.empty(T * N, dtype=torch.int32, device="cuda")
    with capi.CVFilter(N, T, scheme=sch, form=capi.FP64, seed=101, stream=sp) as f:
        f.set_observations_host(ox, oy)
        f.set_ancestry(record_ptr=rec.data_ptr())
        f.initialize()
        f.iterate(T - 1)
        h64 = f.history()
        z64 = f.log_evidence()
    flags = torch.from_numpy(h64["resampled"].astype("int32")).cuda()
    with capi.CVFilter(N, T, scheme=sch, form=capi.MIXED, seed=101, stream=sp) as m:
        m.set_observations_host(ox, oy)
        m.set_ancestry(replay_ptr=rec.data_ptr(), replay_flags_ptr=flags.data_ptr())
        m.initialize()
        m.iterate(T - 1)
        z32 = m.log_evidence()
    del rec
    torch.cuda.synchronize()
    return {"mixed_value": N / (mixed_ms / 1e3), "mixed_ms_per_step": mixed_ms,
            "fp64_ms_per_step": fp64_step_ms, "speedup_mixed_vs_fp64": fp64_step_ms / mixed_ms,
            "mixed_move_ms": mv_ms / n, "log_evidence_fp64": z64, "log_evidence_mixed": z32,
            "rel_log_evidence_error": abs(z32 - z64) / abs(z64),
            "error_method": "mixed run replays the FP64 run's resampling decisions and "
                            "copy_from vectors (fixed ancestry) over the same T steps"}


def mixed_error_sample(capi, cases, scheme=0):
    """The mixed form's error against FP64 for a sample of filters, on a
    fixed ancestry: for each (N, T, ox, oy, seed, stream_id) the FP64 filter
    records its resampling decisions and copy_from vectors and the mixed
    filter replays them.  Batched filters and served requests give the same
    results as the same filter run alone (bit for bit in both forms), so
    this is the error of their results."""
    import numpy as np
    import torch

    errs, rows = [], []
    for (N, T, ox, oy, seed, sid) in cases:
        rec = torch.empty(T * N, dtype=torch.int32, device="cuda")
        with capi.CVFilter(N, T, scheme=scheme, form=capi.FP64, seed=seed,
                           stream_id=sid) as f:
            f.set_observations_host(ox, oy)
            f.set_ancestry(record_ptr=rec.data_ptr())
            f.initialize()
            f.iterate(T - 1)
            h64 = f.history()
            z64 = f.log_evidence()
        flags = torch.from_numpy(h64["resampled"].astype("int32")).cuda()
        with capi.CVFilter(N, T, scheme=scheme, form=capi.MIXED, seed=seed,
                           stream_id=sid) as m:
            m.set_observations_host(ox, oy)
            m.set_ancestry(replay_ptr=rec.data_ptr(),
                           replay_flags_ptr=flags.data_ptr())
            m.initialize()
            m.iterate(T - 1)
            z32 = m.log_evidence()
        del rec
        errs.append(abs(z32 - z64) / abs(z64))
        rows.append({"N": int(N), "T": int(T), "log_evidence_fp64": float(z64),
                     "abs_error": float(abs(z32 - z64))})
    torch.cuda.synchronize()
    worst = int(np.argmax(errs))
    return {"filters": len(errs), "max_rel_log_evidence_error": float(np.max(errs)),
            "median_rel_log_evidence_error": float(np.median(errs)),
            "max_abs_log_evidence_error": float(max(r["abs_error"] for r in rows)),
            "worst": rows[worst],
            "method": "fixed ancestry: the mixed run replays the FP64 run's resampling "
                      "decisions and copy_from vectors"}


def scheme_sweep(capi, sp, sizes=(1 << 16, 1 << 20, 1 << 24), K=20, W=3,
                 cpu=True):
    """Every resampling scheme at N = 2^16, 2^20, 2^24 in both forms: device
    time per step and per move from the library's own CUDA events on the
    filter's stream, over K steps after W warm-up steps of the same filter
    (T = 1 + W + K).  The vSMC reference (StateOMP, all host threads) runs
    the same filter on the host for N <= 2^20."""
    rows = []
    T = 1 + W + K
    ox, oy = capi.cv_simulate(T, OBS_SEED)
    for N in sizes:
        for sch, name in enumerate(SCHEMES):
            row = {"N": N, "scheme": name}
            for form, fname in ((capi.FP64, "fp64"), (capi.MIXED, "mixed")):
                with capi.CVFilter(N, T, scheme=sch, form=form, seed=101, stream=sp) as f:
                    f.set_observations_host(ox, oy)
                    f.initialize()
                    f.iterate(W)
                    f.set_timing(True)
                    f.iterate(K)
                    mv_ms, st_ms, n, _ = f.timing()
                    h = f.history()
                row[fname] = {"ms_per_step": st_ms / n, "move_ms": mv_ms / n,
                              "particle_steps_per_s": N / (st_ms / n / 1e3),
                              "resampled_steps": int(sum(h["resampled"][1 + W:T]))}
            if cpu and N <= 1 << 20:
                v, info = cpu_reference(N, sch, 0, 0, sample_steps=6)
                row["cpu_reference"] = {"particle_steps_per_s": v, "cores": info["cores"],
                                        "kind": info["kind"]}
            rows.append(row)
    return rows


def batched_workload(capi, n_filters=4096, seed=2024):
    """4096 filters: N log-uniform on [2^10, 2^16], T uniform on [50, 500],
    each with its own simulated series (obs seed 1000 + k, stream k)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    N = np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 16), n_filters)).astype(np.int64)
    T = rng.integers(50, 501, n_filters)
    obs = [capi.cv_simulate(int(T[k]), obs_seed=1000 + k, stream_id=k)
           for k in range(n_filters)]
    return N, T, obs


def batched_run(capi, form, N, T, obs, reps=3, autotune=True):
    """Every filter run to the end of its series in one batch: the run is
    one CUDA graph (a step = one launch per kernel over all live filters'
    tiles), at the launch shape the batch's autotuner picks (untimed).
    Device time with CUDA events; e2e adds the observation upload from host
    memory and the log-evidence read back."""
    import numpy as np
    import torch

    nf = len(N)
    psteps = float(np.sum(N * T))
    stream = torch.cuda.Stream()
    with capi.CVBatch(nf, scheme=0, form=form, stream=stream.cuda_stream) as b:
        slots = [b.admit(int(N[k]), int(T[k]), 101 + k, k) for k in range(nf)]
        b.set_observations(slots, obs)
        shape = b.autotune(slots) if autotune else (4, 256)
        b.run(slots)
        b.synchronize()
        dev_ms = []
        for _ in range(reps):
            b.initialize(slots)
            b.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(slots)
            e1.record(stream)
            b.synchronize()
            dev_ms.append(e0.elapsed_time(e1))
        l0 = b.launches()
        b.initialize(slots)
        b.synchronize()
        t0 = time.perf_counter()
        b.set_observations(slots, obs)
        b.run(slots)
        lz = b.read_last(slots)["log_evidence"]
        e2e_s = time.perf_counter() - t0
        launches = b.launches() - l0
    ms = statistics.median(dev_ms)
    return {"filters_per_s": nf / (ms / 1e3), "particle_steps_per_s": psteps / (ms / 1e3),
            "ms_per_run": ms, "e2e_filters_per_s": nf / e2e_s,
            "h2d_bytes": int(16 * np.sum(T)), "d2h_bytes": 40 * nf,
            "gpu_launches_per_run": launches, "log_evidence_first": float(lz[0]),
            "launch_shape": {"move_ctas_per_sm": shape[0], "finalize_threads": shape[1]}}


def serving_requests(lam, seed, max_requests=2000):
    """The request arrivals of one serving point: their number, arrival
    times over min(1 s, max_requests / lam) and sizes N (log-uniform on
    [2^10, 2^18])."""
    import numpy as np

    rng = np.random.default_rng(seed)
    window = min(1.0, max_requests / lam)
    n = max(1, min(max_requests, int(rng.poisson(lam * window))))
    arr = np.sort(rng.uniform(0.0, window, n))
    Ns = np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 18), n)).astype(np.int64)
    return n, arr, Ns


def serving_point(capi, form, lam, seed, T=100, period_s=1e-3, max_requests=2000,
                  budget=16 << 30):
    """Poisson request arrivals at rate `lam`; request N log-uniform on
    [2^10, 2^18]; each streams T observations one at a time, one every
    `period_s` (a 1 kHz sensor).  Latency of an observation = result
    available on the host - its arrival.  Arrivals span min(1 s,
    max_requests / lam)."""
    import numpy as np

    n, arr, Ns = serving_requests(lam, seed, max_requests)
    obs = [capi.cv_simulate(T, obs_seed=5000 + k, stream_id=k) for k in range(n)]
    ox = np.stack([o[0] for o in obs])
    oy = np.stack([o[1] for o in obs])
    # observation k of request r arrives at arr[r] + k * period
    t_obs = (arr[:, None] + period_s * np.arange(T)[None, :]).ravel()
    order = np.argsort(t_obs, kind="stable")
    ev_r = (order // T).astype(np.int64)
    ev_k = (order % T).astype(np.int64)
    ev_t = t_obs[order]
    ids = np.zeros(n, np.uint64)
    opened = np.zeros(n, bool)
    got = []
    n_res = 0
    total = n * T
    with capi.CVServer(4096, scheme=0, form=form, hbm_budget=budget) as srv:
        t0 = srv.now_ns()
        i = 0
        while n_res < total:
            now = (srv.now_ns() - t0) * 1e-9
            j = int(np.searchsorted(ev_t, now, side="right"))
            if j > i:
                rs, ks = ev_r[i:j], ev_k[i:j]
                for r in np.unique(rs[~opened[rs]]):
                    ids[r] = srv.open(int(Ns[r]), T, 101 + int(r), int(r))
                    opened[r] = True
                srv.observe(ids[rs], ox[rs, ks], oy[rs, ks],
                            t0 + (ev_t[i:j] * 1e9).astype(np.int64))
                for r in rs[ks == T - 1]:
                    srv.close(int(ids[r]))
                i = j
            r = srv.poll(wait_ms=0 if i < total else 5)
            if r.size:
                got.append(r)
                n_res += r.size
            elif i < total:
                time.sleep(max(0.0, min(2e-4, ev_t[i] - now)))
        st = srv.stats()
    res = np.concatenate(got)
    lat = (res["done_ns"] - res["submit_ns"]) * 1e-6
    span = (res["done_ns"].max() - res["submit_ns"].min()) * 1e-9
    return {"rate_per_s": lam, "requests": n, "observations": int(total),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "obs_per_s": total / span, "particle_steps_per_s": float(np.sum(Ns) * T / span),
            "ticks": int(st["ticks"]), "max_active": int(st["max_active"]),
            "errors": int(np.sum(res["status"] != 0))}


# Nominal FP32 CUDA-core peak of a B200 (148 SMs x 128 lanes x 2 flops x
# 1965 MHz) and its special-function (exp2 / log2) rate (16 per SM per
# clock); MEASURED_PEAKS.json holds no FP32 figure.
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
SFU_PEAK_TOPS = 148 * 16 * 1.965e9 / 1e12
GMM_FLOPS_PER_POINT = 21  # 4 components x (sub, mul, mul, exp, fma) + log


def gmm_run(capi, form, data, N=1 << 16, iters=100, sweeps=5, seed=101):
    """The tempered SMC sampler (N = 2^16, 100 steps of alpha_t =
    (t/100)^4, 5 sweeps of the three MH block moves, sd 0.1, Systematic at
    ESS < N/2): device time of initialize + all steps, the MCMC kernels'
    share, and their FP32 flop / special-function rates."""
    import torch

    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    with capi.GmmSampler(data, N=N, iters=iters, sweeps=sweeps, form=form, seed=seed,
                         stream=sp) as s:
        s.initialize()  # picks the lanes per particle
        G = s.group()
    with capi.GmmSampler(data, N=N, iters=iters, sweeps=sweeps, form=form, seed=seed,
                         group=G, stream=sp) as s:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.set_timing(True)
        e0.record(stream)
        s.initialize()
        s.iterate(iters)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        mcmc_ms, steps, launches = s.timing()
        logz, path = s.log_evidence()
        h = s.history()
    points = float(N) * iters * 3 * sweeps * len(data)
    flops = points * GMM_FLOPS_PER_POINT
    return {"ms_per_run": ms, "mcmc_ms": mcmc_ms, "lanes_per_particle": G,
            "particle_steps_per_s": N * iters / (ms / 1e3),
            "mcmc_gflops": flops / (mcmc_ms / 1e3) / 1e9,
            "mcmc_fp32_frac_of_nominal": flops / (mcmc_ms / 1e3) / 1e12 / FP32_PEAK_TFLOPS,
            # mixed form: 4 exp2 per point and one log2 per pair of points
            "mcmc_sfu_frac_of_nominal": (4.5 * points / (mcmc_ms / 1e3) / 1e12 / SFU_PEAK_TOPS
                                         if form == capi.MIXED else None),
            "log_evidence": logz, "path_log_evidence": path,
            "resampled_steps": int(h["resampled"].sum()), "gpu_launches": launches}


def gmm_cpu_reference(data, N=2048, iters=100, sweeps=5):
    """vSMC's own example/gmm sampler (oracle/_ref, OpenMP, all threads) on
    the same schedule with fewer particles (the per-particle work does not
    depend on N): particle-steps/s."""
    from oracle import oracle as O

    if not O.gmm_ref_available():
        return None
    r = O.ref_gmm_smc(data, N, iters=iters, sweeps=sweeps)
    return {"value": N * iters / r["seconds"], "unit": "particle-steps/s",
            "cores": O.ref_max_threads(), "kind": "reference",
            "sample": f"vSMC example/gmm sampler, StateOMP, N={N}, {iters} steps, "
                      f"{sweeps} sweeps ({r['seconds']:.1f} s)"}


def run_reference_arm(args):
    rank, world, _ = rank_env()
    if rank != 0:
        return 0
    N = args.particles
    sch = SCHEMES.index(args.scheme)
    T = 1 + args.warmup + args.steps
    v, info = cpu_reference(N, sch, args.warmup, args.steps, threshold=args.threshold)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * N / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (simulated CV Student-t series, Philox4x32-10 seed 7)",
        "config": workload_config(N, T, args.scheme, "fp64", args.threshold, 1,
                                  info["resampled"]),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"],
                         "kind": info["kind"],
                         "sample": f"vSMC Sampler with StateOMP/MoveOMP/MonitorEvalOMP: "
                                   f"initialize + {args.warmup} warm-up + "
                                   f"{args.steps} timed steps at N={N}"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not args.no_state_std:
        # vSMC's std::thread backend on a bounded sample of the same filter
        S = args.cpu_sample_steps
        vs, infs = cpu_reference(N, sch, 0, 0, sample_steps=S, backend=1,
                                 threshold=args.threshold)
        line["state_std"] = {"value": vs, "unit": UNIT, "cores": infs["cores"],
                             "kind": infs["kind"],
                             "sample": f"vSMC StateSTD/MoveSTD (std::thread): initialize "
                                       f"+ {S} steps at N={N}; rate over the {S} steps"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=96)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--particles", type=int, default=1 << 24)
    ap.add_argument("--scheme", default="Multinomial", choices=SCHEMES)
    ap.add_argument("--form", default="fp64", choices=("fp64", "mixed"))
    ap.add_argument("--threshold", type=float, default=0.5,
                    help="resample when ESS < threshold * N (1.1: every step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-state-std", action="store_true",
                    help="skip the StateSTD (std::thread) host baseline")
    ap.add_argument("--cpu-sample-steps", type=int, default=6)
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the form comparison, batched and serving sections")
    ap.add_argument("--serving-rates", default="100,1000,10000,100000")
    ap.add_argument("--gmm-only", choices=("fp64", "mixed"),
                    help="run only the tempered SMC sampler in this form (profiling)")
    ap.add_argument("--gmm-iters", type=int, default=100)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.gmm_only:
        from vsmc_b200 import capi

        capi.lib()
        form = capi.MIXED if args.gmm_only == "mixed" else capi.FP64
        r = gmm_run(capi, form, capi.gmm_simulate(1000, 1), iters=args.gmm_iters)
        print(json.dumps({"workload": f"tempered SMC N=2^16 {args.gmm_iters} steps "
                                      f"{args.gmm_only}", **r}), flush=True)
        return 0

    import numpy as np
    import torch

    from vsmc_b200 import capi
    from vsmc_b200 import replicas

    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    capi.lib()
    N, K, W = args.particles, args.steps, args.warmup
    T = 1 + W + K
    sch = SCHEMES.index(args.scheme)
    form = capi.MIXED if args.form == "mixed" else capi.FP64
    ox, oy = capi.cv_simulate(T, OBS_SEED, stream_id=replicas.replica(rank)["stream_id"])
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, device="cuda")

    rep = replicas.replica(rank)  # this rank's filter: its own counter stream
    f = capi.CVFilter(N, T, scheme=sch, form=form, seed=rep["seed"], threshold=args.threshold,
                      stream_id=rep["stream_id"], stream=sp)
    f.set_observations_host(ox, oy)

    # ---- device-timed run: inputs resident in HBM -------------------------
    f.initialize()
    f.iterate(W)
    f.synchronize()
    clocks = ClockSampler(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    clocks.start()
    time.sleep(0.3)  # let the sampler take a first reading
    with torch.cuda.stream(stream):
        e0.record(stream)
        f.iterate(K)
        f.complete_monitor()  # the last step's monitor, inside the clock
        e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    f.synchronize()
    hist = f.history()
    logz = f.log_evidence()  # of this run (initialize() keeps the engine)
    value = replicas.job_throughput(world, N, K, ms / 1e3)
    resampled = hist["resampled"][1 + W:]
    n_res = int(resampled.sum())

    # ---- kernel timing (library CUDA events on the filter's stream) -------
    f.initialize()
    f.iterate(W)
    f.set_timing(True)
    f.iterate(K)
    move_ms, step_ms, nsteps, launches = f.timing()
    f.set_timing(False)
    f.synchronize()
    peak, peak_kind = load_peaks()
    move_bytes = N * B_MOVE[args.form]
    achieved = move_bytes / (move_ms / nsteps / 1e3) / 1e9
    step_bytes = N * (K * B_MOVE[args.form] + n_res * B_RES[args.form])
    step_achieved = step_bytes / (step_ms / 1e3) / 1e9

    # ---- end to end through the C ABI with host buffers -------------------
    # Streaming use: every step copies its observation from pinned host
    # memory and reads its ESS, increment and flag back to pinned host
    # memory.  The host enqueues step t before it waits for step t-1's
    # result (one step in flight), as a streaming caller would.
    pin_x = torch.from_numpy(ox).pin_memory()
    pin_y = torch.from_numpy(oy).pin_memory()
    outs = torch.zeros((T, 2), dtype=torch.float64).pin_memory()
    ress = torch.zeros(T, dtype=torch.int32).pin_memory()
    done = [torch.cuda.Event() for _ in range(T)]
    g = capi.CVFilter(N, T, scheme=sch, form=form, seed=rep["seed"], threshold=args.threshold,
                      stream_id=rep["stream_id"], stream=sp)
    px, py = pin_x.data_ptr(), pin_y.data_ptr()

    def stream_step(t):
        g.append_observations(px + 8 * t, py + 8 * t, 1)
        g.iterate(1)
        g.read_step(t, outs[t].data_ptr(), outs[t].data_ptr() + 8,
                    ress[t:].data_ptr(), False)
        done[t].record(stream)

    g.append_observations(px, py, 1)
    g.initialize()
    for t in range(1, 1 + W):
        stream_step(t)
        done[t].synchronize()
    barrier()
    t0 = time.perf_counter()
    for t in range(1 + W, T):
        stream_step(t)
        if t > 1 + W:
            done[t - 1].synchronize()  # step t-1's result is on the host
    done[T - 1].synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_logz = g.log_evidence()
    g.close()
    f.close()
    e2e = replicas.job_throughput(world, N, K, e2e_s)

    extras = {}
    if world > 1 and not args.no_extras:
        # filter-partitioned batch: each rank runs its share of the 4096
        # filters in one batch on its own GPU; no collective on the data
        # path; the job's time is the slowest rank's
        bN, bT, bobs = batched_workload(capi)
        parts = replicas.partition_filters([int(n) * int(t) for n, t in zip(bN, bT)], world)
        mine = parts[rank]
        sub = (bN[mine], bT[mine], [bobs[k] for k in mine])
        res = {}
        for fname, fv in (("fp64", capi.FP64), ("mixed", capi.MIXED)):
            barrier()
            r = batched_run(capi, fv, *sub)
            slow_ms = max_over_ranks(r["ms_per_run"])
            res[fname] = {"filters_per_s": len(bN) / (slow_ms / 1e3),
                          "particle_steps_per_s": float(np.sum(bN * bT)) / (slow_ms / 1e3),
                          "ms_per_run": slow_ms, "rank0": r}
        if rank == 0:
            extras["batched"] = {
                "workload": "4096 CV Student-t filters, N log-uniform [2^10, 2^16], T uniform "
                            "[50, 500], Multinomial, threshold 0.5, seeds 101+k, streams k; "
                            f"partitioned over {world} ranks by particle-steps (no collective "
                            "on the data path), time = slowest rank",
                "filters": len(bN), "particle_steps": int(np.sum(bN * bT)),
                "filters_per_rank": [len(p) for p in parts], **res}
    if rank == 0 and world == 1 and not args.no_extras:
        if args.form == "fp64":
            extras["forms"] = forms_compare(capi, N, sch, K, W, ox, oy, sp, ms / K)
        extras["schemes"] = {
            "workload": "CV Student-t filter, each scheme at N = 2^16, 2^20, 2^24, threshold "
                        "0.5, 20 timed steps after 3 warm-up steps",
            "points": scheme_sweep(capi, sp, cpu=not args.no_cpu_baseline)}
        bN, bT, bobs = batched_workload(capi)
        extras["batched"] = {
            "workload": "4096 CV Student-t filters, N log-uniform [2^10, 2^16], T uniform "
                        "[50, 500], Multinomial, threshold 0.5, seeds 101+k, streams k",
            "filters": len(bN), "particle_steps": int(np.sum(bN * bT)),
            "fp64": batched_run(capi, capi.FP64, bN, bT, bobs),
            "mixed": batched_run(capi, capi.MIXED, bN, bT, bobs)}
        b64, b32 = extras["batched"]["fp64"], extras["batched"]["mixed"]
        extras["batched"]["speedup_mixed_vs_fp64"] = b32["filters_per_s"] / b64["filters_per_s"]
        # every 256th filter of the batch (16 filters)
        b32["error_vs_fp64"] = mixed_error_sample(
            capi, [(int(bN[k]), int(bT[k]), bobs[k][0], bobs[k][1], 101 + k, k)
                   for k in range(0, len(bN), 256)])
        gdata = capi.gmm_simulate(1000, 1)
        g64 = gmm_run(capi, capi.FP64, gdata)
        g32 = gmm_run(capi, capi.MIXED, gdata)
        extras["gmm"] = {
            "workload": "tempered SMC, 1-D Gaussian mixture: 1000 points from means "
                        "(-3, 0, 2, 5), N=2^16, 100 steps alpha_t=(t/100)^4, 5 RWMH sweeps "
                        "(mu, log-precision, logit blocks; sd 0.1), Systematic at ESS < N/2",
            "fp64": g64, "mixed": g32,
            "speedup_mixed_vs_fp64": g64["ms_per_run"] / g32["ms_per_run"],
            "roofline": {"bound": "mixed form: special-function units (4 exp2 per point, "
                                  "1 log2 per pair); FP64 form: the FP64 pipe",
                         "peak_fp32_tflops_nominal": FP32_PEAK_TFLOPS,
                         "peak_sfu_tops_nominal": SFU_PEAK_TOPS},
            "cpu_baseline": gmm_cpu_reference(gdata) if not args.no_cpu_baseline else None}
        rates = [float(r) for r in args.serving_rates.split(",") if r]
        extras["serving"] = {
            "workload": "Poisson request arrivals; N log-uniform [2^10, 2^18]; T=100 "
                        "observations per request streamed one every 1 ms; Multinomial; "
                        "HBM budget 16 GiB; latency = result on host - arrival",
            "fp64": [serving_point(capi, capi.FP64, lam, 11) for lam in rates],
            "mixed": [serving_point(capi, capi.MIXED, lam, 11) for lam in rates]}
        # the first 16 requests of the busiest point
        _, _, sNs = serving_requests(max(rates), 11)
        extras["serving"]["mixed_error_vs_fp64"] = mixed_error_sample(
            capi, [(int(sNs[k]), 100) + tuple(capi.cv_simulate(100, obs_seed=5000 + k,
                                                               stream_id=k)) + (101 + k, k)
                   for k in range(min(16, len(sNs)))])

    cpu = None
    # the host reference runs the filter at threshold 0.5
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.threshold == 0.5:
        try:
            S = args.cpu_sample_steps
            v, info = cpu_reference(N, sch, 0, 0, sample_steps=S)
            cpu = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                   "sample": f"vSMC StateOMP, initialize + {S} steps of the same filter "
                             f"at N={N}; rate over the {S} iterate(1) steps"}
            if not args.no_state_std:
                vs, infs = cpu_reference(N, sch, 0, 0, sample_steps=S, backend=1)
                cpu["state_std"] = {
                    "value": vs, "unit": UNIT, "cores": infs["cores"], "kind": infs["kind"],
                    "sample": f"vSMC StateSTD (std::thread), initialize + {S} steps at "
                              f"N={N}"}
        except Exception as ex:  # reported, never silently replaced
            cpu = {"value": None, "unit": UNIT, "cores": None, "kind": None,
                   "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.form == "fp64" else "f32+f64",
            "data": "synthetic (simulated CV Student-t series, Philox4x32-10 seed 7)",
            "config": workload_config(N, T, args.scheme, args.form, args.threshold, world,
                                      n_res),
            "roofline": {"bound": "hbm", "kernel": "k_cv_move",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": load_traffic(args.form, N),
                         "algorithmic_bytes_per_launch": move_bytes,
                         "ms_per_launch": move_ms / nsteps,
                         "step": {"achieved": step_achieved, "frac": step_achieved / peak,
                                  "algorithmic_bytes": step_bytes,
                                  "ms": step_ms}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 16,
                    "d2h_bytes_per_step": 20},
            "gpu_launches": launches,
            "clocks": clk,
            "log_evidence": {"device_run": logz, "e2e_run": e2e_logz},
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
