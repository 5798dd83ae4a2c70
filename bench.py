#!/usr/bin/env python3
"""Benchmark of the B200-native WaveQLab3D per-step volume update.

Workload (one "step" = one low-storage RK time step of the whole block):
plain FP64, one Cartesian block of 101^3 points at h = 0.1 km, homogeneous
elastic medium (Vp 6 km/s, Vs 3.464 km/s, rho 2.67 g/cm^3), traditional
6th-order SBP, free-surface SAT on the q-min face and characteristic
absorbing SAT on the other five, explosive moment-tensor source at the
centre with a Ricker wavelet f0 = 2 Hz, CFL 0.5, a 10 x 10 receiver grid on
the free surface.  The default --steps 500 is the configuration's full run.
Inputs are synthetic (generated here; there is no dataset).

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU
restatement of the reference solver (the Fortran reference needs gfortran
and MPI, which this image lacks) on the host cores instead.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpt-updates/s"
UNIT = "Gpt/s"
WORDS_PER_POINT_STAGE = 39          # F r/w + DF r/w (9 each) + lambda, mu, rho
BYTES_PER_WORD = 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=101)
    return ap.parse_args()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(n):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")) as f:
            t = json.load(f)
        rec = t.get(str(n))
        return None if rec is None else float(rec["dram_bytes_per_launch"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[0]))
                mx = float(s[1])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if s[3 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(problem, target_s=12.0, max_steps=40):
    """Time the CPU oracle (restatement of the reference solver) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    oracle.build()
    d = oracle.OracleDomain(problem)
    npts = problem.blocks[0].npoints
    d.run(1)  # warm-up step
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        d.run(1)
        steps += 1
        if time.perf_counter() - t0 > target_s:
            break
    el = time.perf_counter() - t0
    d.close()
    return {"value": npts * steps / el / 1e9, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port", "sample": f"{steps} RK time steps of the {problem.blocks[0].nqrs[0]}^3 workload "
                                      f"({el:.1f} s, OpenMP over z)"}, el / steps


def run_reference(args, rank, world):
    from waveqlab3d_q_gpu_b200.configs import cartesian_101
    if rank != 0:
        return
    p = cartesian_101(args.n, max(args.steps, 1))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    oracle.build()
    d = oracle.OracleDomain(p)
    npts = p.blocks[0].npoints
    for _ in range(min(args.warmup, 2)):
        d.run(1)
    # each timed step is one RK time step of the workload; the run is capped
    # at about three minutes of CPU time
    t0 = time.perf_counter()
    steps = 0
    while steps < args.steps:
        d.run(1)
        steps += 1
        if time.perf_counter() - t0 > 180.0:
            break
    el = time.perf_counter() - t0
    value = npts * steps / el / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"cartesian-elastic-fp64-{args.n}^3-traditional6-ricker-10x10rec"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": "port",
                         "sample": f"{steps} RK time steps of the {args.n}^3 workload (CPU restatement of the "
                                   f"reference solver; the Fortran reference needs gfortran + MPI, absent here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from waveqlab3d_q_gpu_b200 import build
    build.build()
    from waveqlab3d_q_gpu_b200.configs import cartesian_101
    from waveqlab3d_q_gpu_b200.domain import Domain

    K, W = args.steps, args.warmup
    p = cartesian_101(args.n, K)
    npts = p.blocks[0].npoints
    dt = p.dt()
    g = Domain(p, nsteps_hint=K + W + 4)
    stream = torch.cuda.ExternalStream(g.stream_handle())

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up (also captures the CUDA graph)
    g.run(W)
    g.synchronize()
    barrier()
    l0 = g.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.run(K)
    e1.record(stream)
    g.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = g.kernel_launches() - l0
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * npts * K / (ms / 1e3) / 1e9

    # dominant kernel: the fused stage kernel, timed alone on the library stream
    nst = 40
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for i in range(nst):
        g.stage(1 + i % 4, dt)
    s1.record(stream)
    g.synchronize()
    stage_ms = s0.elapsed_time(s1) / nst
    peak, peak_kind = load_peaks()
    alg_bytes = WORDS_PER_POINT_STAGE * BYTES_PER_WORD * npts
    achieved = alg_bytes / (stage_ms / 1e3) / 1e9
    traffic = load_traffic(args.n)

    # end to end through the public API with pinned host buffers: upload the
    # state, run K steps, read back the seismograms and the final fields
    nq = p.blocks[0].nqrs[0]
    Fh = torch.zeros((9, nq, nq, nq), dtype=torch.float64, pin_memory=True).numpy()
    DFh = torch.zeros((9, nq, nq, nq), dtype=torch.float64, pin_memory=True).numpy()
    g2 = Domain(p, nsteps_hint=K + 4)
    g2.run(2)
    g2.synchronize()
    g2.t = 0.0
    barrier()
    t0 = time.perf_counter()
    g2.set_fields(Fh)
    g2.set_rates_array(DFh)
    g2.run(K)
    seis = g2.seismograms()
    g2.fields(out=Fh)
    g2.synchronize()
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = 2 * Fh.nbytes
    d2h = Fh.nbytes + seis.nbytes
    e2e = {"value": world * npts * K / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
           "d2h_bytes_per_step": d2h / K,
           "what": "set_fields + set_rates from pinned host, run K steps, read seismograms + final fields"}
    g2.close()

    cpu = None
    if rank == 0 and world == 1:
        cpu, _ = cpu_sample(cartesian_101(args.n, K))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"cartesian-elastic-fp64-{args.n}^3-traditional6-ricker-10x10rec",
                       "points": npts, "rk_stages_per_step": 5, "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (state %.0f MB per GPU)" % (g.device_bytes() / 1e6)},
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "k_stage<double,cartesian,elastic>", "stage_ms": stage_ms,
                         "alg_bytes_per_launch": alg_bytes},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
