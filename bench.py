#!/usr/bin/env python3
"""SMC step throughput on B200: the constant-velocity Student-t bootstrap
filter at N = 2^24 particles (BASELINE config 2 shape), one JSON line.

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


def cpu_reference(N, scheme, warmup, steps, sample_steps=None):
    """The vSMC reference (oracle/_ref harness, StateOMP, all host threads) on
    the same filter.  Returns (particle-steps/s over the timed steps, info)."""
    from oracle import oracle as O

    T = 1 + warmup + steps if sample_steps is None else 1 + sample_steps
    ox, oy = O.cv_simulate(T, obs_seed=OBS_SEED)
    if O.ref_available():
        r = O.ref_cv_filter(N, T, scheme, ox, oy, seed=101, backend=0)
        timed = r["step_seconds"][1 + (warmup if sample_steps is None else 0):]
        kind, cores = "reference", O.ref_max_threads()
    else:
        t0 = time.perf_counter()
        O.cv_filter(N, T, scheme, ox, oy, seed=101)
        timed = [time.perf_counter() - t0]
        kind, cores = "port", 1
        T = T
    n_steps = len(timed) if kind == "reference" else T
    return N * n_steps / float(sum(timed)), {"kind": kind, "cores": cores,
                                             "steps": n_steps}


def run_reference_arm(args):
    rank, world, _ = rank_env()
    if rank != 0:
        return 0
    N = args.particles
    sch = SCHEMES.index(args.scheme)
    v, info = cpu_reference(N, sch, args.warmup, args.steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * N / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"cv_student_t N={N} {args.scheme} fp64 "
                               f"threshold 0.5 (vSMC Sampler, StateOMP)",
                   "particles": N, "scheme": args.scheme},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": info["cores"],
                         "kind": info["kind"],
                         "sample": f"initialize + {args.warmup} warm-up + "
                                   f"{args.steps} timed steps at N={N}"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-steps", type=int, default=6)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference_arm(args)

    import numpy as np
    import torch

    from vsmc_b200 import capi

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
    ox, oy = capi.cv_simulate(T, OBS_SEED, stream_id=rank)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    f = capi.CVFilter(N, T, scheme=sch, form=form, seed=101, stream_id=rank, stream=sp)
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
        e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    f.synchronize()
    hist = f.history()
    logz = f.log_evidence()  # of this run (initialize() keeps the engine)
    value = world * N * K / (ms / 1e3)
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
    pin_x = torch.from_numpy(ox).pin_memory()
    pin_y = torch.from_numpy(oy).pin_memory()
    out = torch.zeros(3, dtype=torch.float64).pin_memory()
    res = torch.zeros(1, dtype=torch.int32).pin_memory()
    g = capi.CVFilter(N, T, scheme=sch, form=form, seed=101, stream_id=rank, stream=sp)
    px, py = pin_x.data_ptr(), pin_y.data_ptr()
    g.append_observations(px, py, 1)
    g.initialize()
    for t in range(1, 1 + W):
        g.append_observations(px + 8 * t, py + 8 * t, 1)
        g.iterate(1)
        g.read_step(t, out.data_ptr(), out.data_ptr() + 8, res.data_ptr(), True)
    barrier()
    t0 = time.perf_counter()
    for t in range(1 + W, T):
        g.append_observations(px + 8 * t, py + 8 * t, 1)
        g.iterate(1)
        g.read_step(t, out.data_ptr(), out.data_ptr() + 8, res.data_ptr(), True)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_logz = g.log_evidence()
    g.close()
    f.close()
    e2e = world * N * K / e2e_s

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            S = args.cpu_sample_steps
            v, info = cpu_reference(N, sch, 0, 0, sample_steps=S)
            cpu = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                   "sample": f"vSMC StateOMP, initialize + {S} steps of the same filter "
                             f"at N={N}; rate over the {S} iterate(1) steps"}
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
            "config": {"workload": f"cv_student_t N={N} T={T} {args.scheme} {args.form} "
                                   f"threshold 0.5 seed 101",
                       "particles": N, "scheme": args.scheme, "form": args.form,
                       "resampled_steps": n_res,
                       "l2": "inputs larger than L2 (state 512 MiB FP64 / 256 MiB mixed)",
                       "parallelism": "replicas" if world > 1 else "single"},
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
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
