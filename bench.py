"""Benchmark: laminar 8-block flat plate (228,888 points), FP64, WCNS-E-5
(nscheme 41) + Roe + viscous + LU-SGS, one time step of the reference's loop
(Main.f90:85-109) per timed step.

Prints one JSON line.  Metric: Mcell-steps/s = points x steps / seconds.
  value  -- device-timed: CUDA events around each step's graph replay on the
            library's stream, inputs resident in HBM; L2 flushed between timed
            steps (256 MiB write, outside the timed region).
  e2e    -- the public C ABI with host buffers: per step the prim state of
            every block is copied in from pinned host memory
            (wcns_set_prim_all, ghosted layout), the step runs (wcns_step),
            and the resulting interior state (wcns_get_flow, flow-file
            layout) and the residual (wcns_residual) are copied back.
  --impl reference -- the CPU restatement of the reference path (the oracle;
            the Fortran reference cannot be built here) on all host cores.
N>1 (torchrun): every rank runs its own replica of the case (weak scaling);
timing is the max over ranks.
"""
from __future__ import annotations

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

METRIC = "Mcell-steps/s"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# algorithmic bytes per point-step (FP64 words x 8): RHS 20, LU-SGS L 25,
# U 25, GS-L 30, GS-U 30, update+residual 15 words (1,160 B per point-step)
WORDS = {"rhs": 20, "lhs": 110, "update": 15, "step": 145}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--case", default="plate")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10)
    return ap.parse_args()


def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = os.environ.get("WCNS_DIST_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": len(self.samples)}
        if not self.samples:
            return out
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        out.update(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=sorted(reasons))
        return out


def load_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_step_traffic(npoints):
    """DRAM bytes (read + write) of one time step, summed over the step's
    kernels from an ncu capture of the plate workload, scaled per point;
    None when no capture summary is present."""
    path = os.path.join(ROOT, "profiles", "plate_step_dram.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_point_step:"):
                return int(float(line.split(":")[1]) * npoints)
    except OSError:
        pass
    return None


def make_case(name):
    from wcns_b200 import cases
    if name == "plate":
        return cases.plate_case()
    if name == "vortex":
        return cases.vortex_case()
    return cases.CASES[name]()


def cpu_reference_rate(case, steps, threads=None, target_s=None):
    """Oracle (CPU restatement) throughput on `steps` full steps of `case`
    after one untimed step; with `target_s`, the number of steps is chosen
    from the untimed step so that the timed sample lasts about that long."""
    from oracle.pyoracle import Oracle
    o = Oracle(case, nthreads=threads or os.cpu_count())
    t0 = time.perf_counter()
    o.step(1)
    one = time.perf_counter() - t0
    if target_s:
        steps = int(min(200, max(steps, round(target_s / max(one, 1e-3)))))
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    o.close()
    return case.npoints * steps / dt / 1e6, dt, steps


def run_reference(args, rank, world):
    if rank != 0:
        return
    case = make_case(args.case)
    cores = os.cpu_count()
    # each step is one full step of the workload on all host cores
    rate, dt, _ = cpu_reference_rate(case, max(1, args.steps), cores)
    line = {
        "metric": METRIC, "value": round(rate, 4), "unit": "Mcell-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * dt / max(1, args.steps), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"{case.name}: {case.description}", "points": case.npoints, "blocks": case.nblocks},
        "cpu_baseline": {"value": round(rate, 4), "unit": "Mcell-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full steps of the workload after 1 untimed step (OpenMP over blocks/lines)"},
        "e2e": {"value": round(rate, 4), "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_b200(args, rank, world):
    import numpy as np
    import torch

    from wcns_b200.solver import Wcns
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    case = make_case(args.case)
    g = Wcns(case)
    stream = torch.cuda.ExternalStream(g.stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # warm-up
    g.step(args.warmup, history=False)
    dist_barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    evs = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        g.step_async(1)
        e1.record(stream)
        evs.append((e0, e1))
    g.sync()
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    clk = clocks.stop()
    dist_barrier(world)
    ms = dist_max(ms, world)
    total_points = case.npoints * world
    value = total_points * args.steps / (ms / 1e3) / 1e6

    # Roofline of the step program: one graph replay = one step of the whole
    # path.  Algorithmic bytes = the compulsory traffic of one point-step
    # (WORDS["step"] FP64 words: each globally dependent phase reads its
    # inputs once and writes its outputs once) x points; duration = the
    # CUDA-event time of the timed steps above.
    peak, peak_kind = load_peak()
    step_bytes = case.npoints * WORDS["step"] * 8
    achieved = step_bytes / (ms / args.steps / 1e3) / 1e9
    traffic = load_step_traffic(case.npoints)

    # end-to-end through the C ABI with pinned host buffers
    pinned = []
    for nb, d in enumerate(case.dims, start=1):
        ni, nj, nk = d
        bufs = [torch.empty((nk + 6, nj + 6, ni + 6), dtype=torch.float64, pin_memory=True).numpy() for _ in range(6)]
        for f, name in enumerate(("r", "u", "v", "w", "p", "t")):
            bufs[f][...] = g.get(name, nb)
        pinned.append(bufs)
    # results: the interior state of every block in the flow-file layout
    outs = [[torch.empty((nk, nj, ni), dtype=torch.float64, pin_memory=True).numpy() for _ in range(5)]
            for ni, nj, nk in case.dims]
    h2d = sum(6 * a[0].size * 8 for a in pinned)
    d2h = sum(5 * a[0].size * 8 for a in outs) + 8 * (2 * case.nblocks + 1)
    dist_barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        g.set_prim_all(pinned)
        g.step(1, history=False)
        g.get_flow(outs)
        g.residual_curve()
    e2e_s = time.perf_counter() - t0
    e2e_s = dist_max(e2e_s, world)
    e2e = total_points * args.e2e_steps / e2e_s / 1e6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, dt, n = cpu_reference_rate(case, 3, os.cpu_count(), target_s=10.0)
            cpu = {"value": round(rate, 4), "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"{n} full steps of the workload after 1 untimed step ({dt:.1f} s, OpenMP)"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {e}"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "Mcell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"{case.name}: {case.description}", "points": case.npoints,
                       "blocks": case.nblocks, "nscheme": case.params.nscheme, "nflux": case.params.nflux,
                       "l2": "256 MiB flush between timed steps", "parallelism": f"replicas x{world}"},
            "e2e": {"value": round(e2e, 4), "unit": "Mcell-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "kernel": "one time step (CUDA graph of the whole path)",
                         "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 5), "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": int(step_bytes), "launch_ms": round(ms / args.steps, 4),
                         "traffic": traffic},
            "gpu_launches": g.launches_per_step() * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    rank, world = dist_init(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return
    run_b200(args, rank, world)


if __name__ == "__main__":
    main()
