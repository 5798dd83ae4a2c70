#!/usr/bin/env python3
"""Benchmark of the B200-native WaveQLab3D per-step volume update.

Default workload (``--workload hill``): the curvilinear two-block Q8 + PML
problem.  A 201 x 201 x 201-point domain at h = 0.05 km split at mid-depth
into two 101 x 201 x 201 blocks joined by a locked q-interface; Gaussian-hill
topography (0.8 km, sigma 2.5 km) with seeded random bumps; Vs layered
2.0 -> 3.5 km/s, Vp = sqrt(3) Vs, rho = 1.7 + 0.2 Vp; Q8 with per-point
Qs = 50 Vs, Qp = 2 Qs; free surface on top, 20-point PML on the sides and
bottom; seeded double-couple with a Ricker wavelet f0 = 3 Hz; 10 x 10
surface stations.  One "step" is one five-stage low-storage RK time step of
both blocks and the interface.  The plain FP64 path gives ``value``; the
FP32 path with compensated state accumulation is measured on the same
workload and reported under ``fp32`` with its seismogram error against FP64.

``--workload cartesian`` times the plain FP64 single Cartesian 101^3 block
(explosive Ricker source, free surface on the q-min face) instead;
``--workload planar`` the two-block 512 x 512 x 384 Cartesian planar
slip-weakening fault with fQ8 in a von Karman medium (its CPU leg runs a
128 x 128 x 96 instance of the same workload).  ``--workload shots`` runs the batched
independent shots (48 Cartesian elastic / Q4 problems of 64^3 - 192^3 points,
seeded media, sources and Ricker frequencies) concurrently on one device in
FP32, checked against FP64 solves of the same shots.

Inputs are synthetic (generated here; there is no dataset).  Prints one JSON
line (rank 0).  ``--impl reference`` times the CPU restatement of the
reference solver on the host cores (the Fortran reference needs gfortran and
MPI, which this image lacks).
"""
import argparse
import json
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="hill", choices=["hill", "cartesian", "planar", "shots"])
    ap.add_argument("--nshots", type=int, default=48, help="shots of --workload shots")
    ap.add_argument("--n", type=int, default=None, help="points per axis (201 hill, 101 cartesian)")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--only-fp32", action="store_true", help="time the FP32 path alone (profiling)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend of N > 1 runs (gloo: host-side swaps, e.g. two ranks on one GPU)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint / forward ratio leg")
    ap.add_argument("--adjoint-steps", type=int, default=64, help="steps of the adjoint ratio leg")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the full-duration FP32 accuracy leg")
    ap.add_argument("--accuracy-steps", type=int, default=750, help="steps of the FP32 accuracy leg")
    return ap.parse_args()


def make_problem(args, steps, cpu_sample=False):
    from waveqlab3d_q_gpu_b200.configs import cartesian_101, hill_two_block_q8, planar_fault_fq8
    if args.workload == "shots":
        from waveqlab3d_q_gpu_b200.shots import random_shot
        return random_shot(7000, steps=steps), "batched-shots-one-shot-sample"
    if args.workload == "cartesian":
        n = args.n or 101
        return cartesian_101(n, steps), f"cartesian-elastic-fp64-{n}^3-traditional6-ricker-10x10rec"
    if args.workload == "planar":
        n = 128 if cpu_sample else (args.n or 512)
        ns = 3 * n // 4
        return (planar_fault_fq8(n, n, ns, steps=steps),
                f"planar-fault-2block-{n}x{n}x{ns}-fq8-vonkarman-slipweakening")
    n = args.n or 201
    return (hill_two_block_q8(n, steps=steps),
            f"curvilinear-2block-{n}^3-hill-q8-pml20-locked-ricker3hz-10x10rec")


def words_per_stage(problem):
    """Algorithmic words per RK stage, summed over all points: F r/w and DF r/w
    (36), lambda mu rho (3), curvilinear metric + J (10), Q4/Q8 memory
    variables and their rates read and written (24 per mechanism) + Qs^-1,
    Qp^-1 (2), fQ8 (24 per mechanism), 36 per PML slab a point lies in.
    Ghost cells, halo re-reads and the O(n^2) face / interface / source terms
    are not counted."""
    per_pt = 36 + 3
    if problem.type_of_mesh == "curvilinear":
        per_pt += 10
    nm = problem.nmech
    if problem.response in ("anelastic-Q4", "anelastic-Q8"):
        per_pt += 24 * nm + 2
    elif problem.response == "anelastic-fQ8":
        per_pt += 24 * nm
    total = 0
    for b in problem.blocks:
        nq, nr, ns = b.nqrs
        total += per_pt * b.npoints
        if b.npml > 0:
            face = {0: nr * ns, 1: nq * ns, 2: nq * nr}
            for f, on in enumerate(b.pml()):
                if on:
                    total += 36 * b.npml * face[f // 2]
    return total


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(key):
    """(DRAM bytes per RK stage of the stage kernels, how they were measured)
    from the committed ncu summary, or (None, None)."""
    try:
        with open(os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")) as f:
            t = json.load(f)
        rec = t.get(key)
        return (None, None) if rec is None else (float(rec["dram_bytes_per_stage"]), rec.get("how"))
    except Exception:
        return None, None


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


def oracle_steps(problem, steps, warmup, budget_s):
    """Time the CPU oracle (restatement of the reference solver, OpenMP over
    z) for at most ``steps`` time steps or ``budget_s`` seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    oracle.build()
    d = oracle.OracleDomain(problem)
    for _ in range(warmup):
        d.run(1)
    n, t0 = 0, time.perf_counter()
    while n < steps:
        d.run(1)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    d.close()
    npts = sum(b.npoints for b in problem.blocks)
    return npts * n / el / 1e9, n, el, int(os.environ["OMP_NUM_THREADS"])


STEPS_OF_CONFIG = {"hill": 1500, "cartesian": 500, "planar": 2000}


def workload_config(args, name, npts, nblocks, world):
    """The line's ``config``: what the workload is and how it is spread over the
    N processes, identical in both arms (the timing details sit outside it)."""
    if world > 1 and world % 2 == 0 and args.workload == "hill":
        return {"workload": name, "points_per_copy": npts, "copies": world // 2,
                "parallelism": f"blocks2x{world // 2}", "backend": args.dist_backend,
                "exchange": "interface face trace every RK stage, NCCL send/recv into the library's receive buffer"}
    return {"workload": name, "points": npts, "blocks": nblocks, "rk_stages_per_step": 5,
            "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (126 MB) at every step"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    p, name = make_problem(args, max(args.steps, 1), cpu_sample=True)
    if args.workload == "planar":
        # the configuration is the full-size one (two blocks of n/2 x n x 3n/4);
        # the CPU times its 128 x 128 x 96 instance
        n = args.n or 512
        cfg = workload_config(args, f"planar-fault-2block-{n}x{n}x{3 * n // 4}-fq8-vonkarman-slipweakening",
                              n * n * (3 * n // 4), 2, world)
    else:
        cfg = workload_config(args, name, sum(b.npoints for b in p.blocks), len(p.blocks), world)
    value, n, el, cores = oracle_steps(p, args.steps, min(args.warmup, 1), 150.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": n,
        "warmup": args.warmup, "ms_per_step": 1e3 * el / n, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{n} RK time steps of the workload in {el:.1f} s (CPU restatement of the "
                                   f"reference solver, OpenMP over z; the Fortran reference needs gfortran + MPI, "
                                   f"absent here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed_run(g, stream, K, barrier):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    g.run(K)
    e1.record(stream)
    g.synchronize()
    barrier()
    return e0.elapsed_time(e1)


def stage_time(g, stream, dt, nst=20):
    """Average duration of one RK stage (both blocks' stage kernels and the
    interface kernel) on the library stream."""
    import torch
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    g.stage(2, dt)
    s0.record(stream)
    for i in range(nst):
        g.stage(2 + i % 4, dt)
    s1.record(stream)
    g.synchronize()
    return s0.elapsed_time(s1) / nst


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
    torch.cuda.set_device(local % max(1, torch.cuda.device_count()))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(args.dist_backend, timeout=datetime.timedelta(seconds=120))
    from waveqlab3d_q_gpu_b200 import build
    build.build()
    from waveqlab3d_q_gpu_b200.domain import Domain

    K, W = args.steps, max(args.warmup, 3)
    p, name = make_problem(args, K + W + 4) if args.workload != "shots" else (None, None)
    npts = sum(b.npoints for b in p.blocks) if p is not None else 0
    nb = len(p.blocks) if p is not None else 0

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda" if args.dist_backend == "nccl" else "cpu", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if world > 1 and world % 2 == 0 and args.workload == "hill":
        pairs_main(args, rank, world, local, barrier, max_over_ranks, p, name)
        dist.barrier()
        dist.destroy_process_group()
        return

    if args.workload == "shots":
        shots_main(args, rank, world, local, barrier, max_over_ranks)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    peak, peak_kind = load_peaks()
    words = words_per_stage(p)
    results = {}
    precisions = ["fp64"] if args.no_fp32 else (["fp32"] if args.only_fp32 else ["fp64", "fp32"])
    clk = None
    for prec in precisions:
        g = Domain(p, precision=prec, nsteps_hint=K + W + 4)
        stream = torch.cuda.ExternalStream(g.stream_handle())
        g.run(W)                      # warm-up, captures the CUDA graph
        g.synchronize()
        l0 = g.kernel_launches()
        clocks = ClockSampler(local) if prec == "fp64" else None
        if clocks:
            clocks.start()
        ms = timed_run(g, stream, K, barrier)
        if clocks:
            clk = clocks.stop()
        launches = g.kernel_launches() - l0
        ms = max_over_ranks(ms)
        seis = g.seismograms(0)
        fields = [g.fields(bi) for bi in range(len(p.blocks))] if "fp32" in precisions else None
        st_ms = stage_time(g, stream, p.dt())
        w = 8 if prec == "fp64" else 4
        achieved = words * w / (st_ms / 1e3) / 1e9
        results[prec] = {"ms_per_step": ms / K, "value": world * npts * K / (ms / 1e3) / 1e9,
                         "launches": int(launches), "stage_ms": st_ms, "achieved": achieved, "seis": seis,
                         "fields": fields, "bytes": g.device_bytes()}
        g.close()
        del g
        torch.cuda.empty_cache()
    if "fp64" not in results:
        r = results["fp32"]
        print(json.dumps({"metric": METRIC, "value": r["value"], "unit": UNIT, "dtype": "f32",
                          "ms_per_step": r["ms_per_step"], "stage_ms": r["stage_ms"],
                          "config": {"workload": name}, "note": "FP32 path alone (profiling run)"}), flush=True)
        return
    r64 = results["fp64"]

    # end to end through the public API with pinned host buffers: upload the
    # initial fields of both blocks, run K steps, read back the stations and
    # the final fields of both blocks
    hosts = []
    for b in p.blocks:
        nq, nr, ns = b.nqrs
        hosts.append(torch.zeros((9, ns, nr, nq), dtype=torch.float64, pin_memory=True).numpy())
    g2 = Domain(p, nsteps_hint=K + 4)
    g2.run(2)
    g2.synchronize()
    g2.t = 0.0
    barrier()
    t0 = time.perf_counter()
    for bi in range(nb):
        g2.set_fields(hosts[bi], bi)
    g2.run(K)
    seis2 = g2.seismograms(0)
    for bi in range(nb):
        g2.fields(bi, out=hosts[bi])
    g2.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    h2d = sum(h.nbytes for h in hosts)
    d2h = sum(h.nbytes for h in hosts) + seis2.nbytes
    e2e = {"value": world * npts * K / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
           "d2h_bytes_per_step": d2h / K,
           "what": "set_fields of both blocks from pinned host, run K steps, read stations + final fields"}
    g2.close()
    del g2

    adj = adjoint_leg(args, barrier) if (args.workload == "hill" and not args.no_adjoint) else None
    acc = fp32_accuracy_leg(args) if (args.workload == "hill" and "fp32" in results and not args.no_accuracy) else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        pc, cname = (p, name) if args.workload != "planar" else make_problem(args, 4, cpu_sample=True)
        v, n, el, cores = oracle_steps(pc, 2, 0, 30.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{n} RK time step(s) of {cname} in {el:.1f} s (CPU restatement of the "
                         f"reference solver, OpenMP over z)"}

    if rank == 0:
        traffic, traffic_how = load_traffic(name)
        line = {
            "metric": METRIC, "value": r64["value"], "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": r64["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, name, npts, nb, world),
            "device_bytes": r64["bytes"],
            "timed_steps_of_run": f"{K} of the configuration's {STEPS_OF_CONFIG.get(args.workload, '?')}",
            "e2e": e2e,
            "gpu_launches": r64["launches"],
            "roofline": {"bound": "hbm", "achieved": r64["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": r64["achieved"] / peak, "traffic": traffic, "traffic_how": traffic_how,
                         "peak_kind": peak_kind,
                         "kernel": "one RK stage: stage kernels of both blocks + interface kernel",
                         "stage_ms": r64["stage_ms"], "alg_bytes_per_stage": words * 8},
            "cpu_baseline": cpu,
            "clocks": clk,
        }
        if adj is not None:
            line["adjoint"] = adj
        if acc is not None:
            line["fp32_accuracy"] = acc
        if "fp32" in results:
            r32 = results["fp32"]
            s64, s32 = r64["seis"][:, :, 1:], r32["seis"][:, :, 1:]
            err = float(np.linalg.norm(s32 - s64) / max(np.linalg.norm(s64), 1e-300))
            num = sum(float(np.linalg.norm(a - b) ** 2) for a, b in zip(r32["fields"], r64["fields"]))
            den = sum(float(np.linalg.norm(b) ** 2) for b in r64["fields"])
            ferr = (num / max(den, 1e-300)) ** 0.5
            line["fp32"] = {"value": r32["value"], "ms_per_step": r32["ms_per_step"],
                            "speedup_vs_fp64": r32["value"] / r64["value"],
                            "roofline": {"achieved": r32["achieved"], "frac": r32["achieved"] / peak,
                                         "stage_ms": r32["stage_ms"], "alg_bytes_per_stage": words * 4,
                                         "note": "compensation array (+18 words/pt/stage) not counted"},
                            "seismogram_rel_l2_vs_fp64": err, "fields_rel_l2_vs_fp64": ferr,
                            "error_note": "after the warm-up and timed steps; short runs end before the direct "
                                          "wave reaches the surface stations, so the field error is the meaningful one",
                            "gpu_launches": r32["launches"]}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def pairs_main(args, rank, world, local, barrier, max_over_ranks, p, name):
    """N = 2, 4, 6, 8 GPUs: the two-block workload with one block per GPU, as
    the reference runs it (one MPI rank per block): ranks 2k and 2k + 1 hold
    blocks 1 and 2 of one copy of the problem and swap the interface face
    trace every RK stage over NCCL into the library's receive buffer
    (distributed.BlockRank).  N / 2 copies run side by side (weak scaling over
    copies, each copy split over two GPUs).  Timed with CUDA events on each
    rank's domain stream between barriers, max over ranks."""
    import numpy as np
    import torch
    from waveqlab3d_q_gpu_b200.distributed import BlockRank
    K, W = args.steps, max(args.warmup, 3)
    block, peer = rank % 2, rank ^ 1
    npts = sum(b.npoints for b in p.blocks)
    br = BlockRank(p, block, backend=args.dist_backend, nsteps_hint=K + W + 4, peer=peer)
    g = br.domain
    stream = torch.cuda.ExternalStream(g.stream_handle())
    br.run(W)
    g.synchronize()
    l0 = g.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    br.run(K)
    e1.record(stream)
    g.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1))
    launches = g.kernel_launches() - l0
    # end to end: this rank's block from pinned host, K steps, stations and fields back
    nq, nr, ns = p.blocks[block].nqrs
    host = torch.zeros((9, ns, nr, nq), dtype=torch.float64, pin_memory=True).numpy()
    barrier()
    t0 = time.perf_counter()
    g.set_fields(host, 0)
    br.run(K)
    seis = g.seismograms(0)
    g.fields(0, out=host)
    g.synchronize()
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    br.close()
    copies = world // 2
    if rank == 0:
        line = {"metric": METRIC, "value": copies * npts * K / (ms / 1e3) / 1e9, "unit": UNIT, "n_gpus": world,
                "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(args, name, npts, len(p.blocks), world),
                "e2e": {"value": copies * npts * K / e2e_s / 1e9, "unit": UNIT,
                        "h2d_bytes_per_step": world * host.nbytes / K,
                        "d2h_bytes_per_step": world * (host.nbytes + seis.nbytes) / K,
                        "what": "every rank's block from pinned host, K steps, stations + final fields back"},
                "gpu_launches": int(launches) * world, "roofline": None, "cpu_baseline": None, "clocks": clk}
        print(json.dumps(line), flush=True)


def fp32_accuracy_leg(args):
    """Seismogram error of the FP32 compensated path against FP64 over the whole
    duration of the curvilinear two-block Q8 + PML workload: the same 10 km
    domain, hill, media, source and stations at h = 0.1 km (101^3 points), run
    for the configuration's 1500 steps of h = 0.05 km (750 steps at the
    doubled time step), so the direct wave and the surface waves reach every
    station.  Relative L2 over all stations and samples, and the worst station."""
    import numpy as np
    from waveqlab3d_q_gpu_b200.configs import hill_two_block_q8
    from waveqlab3d_q_gpu_b200.domain import Domain
    steps = args.accuracy_steps
    p = hill_two_block_q8(101, h=0.1, steps=steps)
    seis = {}
    for prec in ("fp64", "fp32"):
        g = Domain(p, precision=prec, nsteps_hint=steps + 2)
        g.run(steps)
        seis[prec] = g.seismograms(0)[:, :, 1:]
        g.close()
    a, b = seis["fp32"], seis["fp64"]
    err = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    per = [float(np.linalg.norm(a[:, r] - b[:, r]) / max(np.linalg.norm(b[:, r]), 1e-300)) for r in range(b.shape[1])]
    return {"workload": "curvilinear-2block-101^3-h0.1-hill-q8-pml20-locked-ricker3hz-10x10rec (same domain and "
                        "physics as the timed workload at half the resolution)",
            "steps": steps, "seismogram_rel_l2_vs_fp64": err, "worst_station_rel_l2": max(per),
            "median_station_rel_l2": float(np.median(per)), "peak_velocity": float(np.abs(b).max())}


def adjoint_leg(args, barrier):
    """Adjoint / forward time ratio on the gradient configuration's grid
    (configs.adjoint_block: curvilinear 201 x 201 x 101 at h = 0.1 km, elastic,
    one source, 20 x 20 surface stations) over a sample of the run: one
    forward solve with sqrt(N) checkpoints versus the reverse sweep that
    recomputes the segments and applies the adjoint steps, both timed on the
    device stream with a synchronize on both sides.  The misfit compares with
    data of the true model (3 % Vs anomaly)."""
    import numpy as np
    import torch
    from waveqlab3d_q_gpu_b200.adjoint import AdjointSolver
    from waveqlab3d_q_gpu_b200.configs import adjoint_block
    N = args.adjoint_steps
    true = adjoint_block(anomaly=True, steps=N)
    sol = AdjointSolver(true, N)
    observed = sol.forward()
    sol.set_parameters(material=adjoint_block(anomaly=False, steps=N).blocks[0].material)
    sol.forward()
    sol.backward(np.zeros_like(observed))           # warm-up (graphs, first launches)
    barrier()
    t0 = time.perf_counter()
    seis = sol.forward()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    gmat, gM = sol.backward(seis - observed)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    fwd, bwd = t1 - t0, t2 - t1
    npts = true.blocks[0].npoints
    sol.close()
    return {"workload": "curvilinear-201x201x101-h0.1-elastic-1src-20x20rec (gradient configuration grid; "
                        "discrete adjoint covers elastic blocks without PML)",
            "steps": N, "checkpoint_every": sol.K, "forward_s": fwd, "backward_s": bwd,
            "adjoint_forward_ratio": (fwd + bwd) / fwd, "backward_forward_ratio": bwd / fwd,
            "forward_gpt_s": npts * N / fwd / 1e9,
            "gradient_norms": {"material": float(np.linalg.norm(gmat)), "moment": float(np.linalg.norm(gM))}}


def shots_main(args, rank, world, local, barrier, max_over_ranks):
    """Batched shots: every shot a domain on its own stream, replayed
    round-robin; the timed region spans all streams (each stream's end event
    joins the first stream before the stop event)."""
    import numpy as np
    import torch
    from waveqlab3d_q_gpu_b200.shots import ShotBatch, random_shots
    K, W = args.steps, max(args.warmup, 3)
    ps = random_shots(args.nshots, seed=7 + rank, steps=K + W + 4)
    name = f"batched-shots-{args.nshots}x(64..192)^3-elastic-q4-ricker1-4hz"
    npts = sum(b.npoints for q in ps for b in q.blocks)
    words = sum(words_per_stage(q) for q in ps)
    peak, peak_kind = load_peaks()

    def timed(batch, nsteps):
        streams = [torch.cuda.ExternalStream(d.stream_handle()) for d in batch.domains]
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        for s in streams[1:]:
            s.wait_event(e0)
        batch.run(nsteps)
        for s in streams[1:]:
            ev = torch.cuda.Event()
            ev.record(s)
            streams[0].wait_event(ev)
        e1.record(streams[0])
        batch.synchronize()
        barrier()
        return e0.elapsed_time(e1)

    res = {}
    clk = None
    for prec in ("fp32", "fp64", "fp32-streams"):
        mode = "streams" if prec.endswith("streams") else "batched"
        batch = ShotBatch(ps, precision=prec[:4], nsteps_hint=W + 2 * K + 10, mode=mode)
        batch.run(max(W, 8))           # warm-up; the batched mode's tile autotuner uses its first 6 steps
        batch.synchronize()
        l0 = batch.kernel_launches()
        clocks = ClockSampler(local) if prec == "fp32" else None
        if clocks:
            clocks.start()
        ms = max_over_ranks(timed(batch, K))
        if clocks:
            clk = clocks.stop()
        launches = batch.kernel_launches() - l0
        res[prec] = {"ms": ms, "value": world * npts * K / (ms / 1e3) / 1e9, "launches": int(launches),
                     "seis": batch.seismograms(), "bytes": sum(d.device_bytes() for d in batch.domains),
                     "tuning": batch.tuning() if mode == "batched" else None}
        if prec == "fp32-streams":
            batch.close()
            del batch
            torch.cuda.empty_cache()
            continue
        if prec == "fp32":
            # end to end: each shot's initial fields from pinned host, run, stations back
            hosts = [torch.zeros((9,) + tuple(q.blocks[0].nqrs[::-1]), dtype=torch.float64,
                                 pin_memory=True).numpy() for q in ps]
            for d in batch.domains:
                d.t = 0.0
            barrier()
            t0 = time.perf_counter()
            for d, hbuf in zip(batch.domains, hosts):
                d.set_fields(hbuf, 0)
            batch.run(K)
            seis_e2e = batch.seismograms()
            batch.synchronize()
            barrier()
            el = time.perf_counter() - t0
            e2e = {"value": world * npts * K / el / 1e9, "unit": UNIT,
                   "h2d_bytes_per_step": sum(h.nbytes for h in hosts) / K,
                   "d2h_bytes_per_step": sum(x.nbytes for x in seis_e2e) / K,
                   "what": "set_fields of every shot from pinned host, run K steps, read every shot's stations"}
        batch.close()
        del batch
        torch.cuda.empty_cache()
    # per-shot station error of FP32 against FP64, over the shots whose
    # stations the direct wave has reached within the run
    norms = [float(np.linalg.norm(b[:, :, 1:])) for b in res["fp64"]["seis"]]
    big = max(norms) if norms else 0.0
    errs = [float(np.linalg.norm(a[:, :, 1:] - b[:, :, 1:]) / nb)
            for a, b, nb in zip(res["fp32"]["seis"], res["fp64"]["seis"], norms) if nb > 1e-6 * big]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, n, el, cores = oracle_steps(ps[0], 2, 0, 30.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{n} RK time step(s) of shot 0 ({'x'.join(map(str, ps[0].blocks[0].nqrs))}) in "
                         f"{el:.1f} s (CPU restatement of the reference solver, OpenMP over z)"}
    if rank == 0:
        r = res["fp32"]
        achieved = words * 4 * 5 * K / (r["ms"] / 1e3) / 1e9
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
                "ms_per_step": r["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": name, "shots": len(ps), "points": npts, "parallelism": f"replicas{world}",
                           "l2": "inputs larger than L2 (%.1f GB on the device)" % (r["bytes"] / 1e9)},
                "e2e": e2e, "gpu_launches": r["launches"],
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                             "kernel": "whole step of every shot (stage kernels, concurrent streams)",
                             "alg_bytes_per_step": words * 4 * 5},
                "cpu_baseline": cpu, "clocks": clk,
                "fp64": {"value": res["fp64"]["value"], "ms_per_step": res["fp64"]["ms"] / K},
                "batched": {"launches_per_step": r["launches"] / K, "zchunk": r["tuning"][0],
                            "tuning_ms_per_step": {str(z): m for z, m in r["tuning"][1]},
                            "what": "one launch per kernel kind and RK stage for all shots, two-step CUDA graph"},
                "streams": {"value": res["fp32-streams"]["value"], "ms_per_step": res["fp32-streams"]["ms"] / K,
                            "launches_per_step": res["fp32-streams"]["launches"] / K,
                            "what": "each shot its own stream and step graph, replayed round-robin"},
                "seismogram_rel_l2_fp32_vs_fp64": {"max": max(errs) if errs else None,
                                                   "median": float(np.median(errs)) if errs else None,
                                                   "shots_with_signal": len(errs)}}
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
