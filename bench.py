"""Benchmark: the SA turbulent channel with a Gaussian wall bump (24 blocks of
seeded uneven sizes, 4,157,400 points, Re_H 5e6, Mach 0.6), FP64, WCNS-E-5
(nscheme 41) + Roe + viscous + Spalart-Allmaras + LU-SGS, one time step of
the reference's loop (Main.f90:85-109) per timed step.  `--case plate` runs
the laminar 8-block flat plate (228,888 points) instead.

Prints one JSON line.  Metric: Mcell-steps/s = points x steps / seconds.
  value  -- device-timed: CUDA events on the library's stream around K graph
            replays (one replay = one whole step), inputs resident in HBM.
            The channel's resident fields (about 11 GB) are far larger than
            L2, so steps run back to back; a workload smaller than 4x L2 is
            timed step by step with a 256 MiB L2 flush between steps (outside
            the timed region).
  phases -- one extra step enqueued phase by phase with CUDA events between
            the phases (wcns_profile_step), outside the timed region: device
            ms and share of every phase, the LU-SGS sweeps separately.
  e2e    -- the public C ABI with host buffers: per step the interior state
            of every block (r, u, v, w, p and, with the SA model, qke) is
            copied in from pinned host memory (wcns_set_interior, flow-file
            layout), the step runs (wcns_step), the same fields are copied
            back (wcns_get_interior) and the residual read (wcns_residual).
  mixed_precision -- (one GPU) the same workload with the mixed-precision
            residual (wcns_set_precision 32): Mcell-steps/s, speed-up over
            the FP64 line, per-variable relative L2 and wall-force errors
            against a fresh FP64 context after the same steps.
  batch64 -- (one GPU) 64 independent small SA bump cases: every case on
            its own FP64 context one after another, all in one FP64
            context, all in one context with the mixed-precision residual;
            Mcell-steps/s of each, speed-ups, errors of the mixed batch.
  --impl reference -- the CPU restatement of the reference path (the oracle;
            the Fortran reference cannot be built here) on all host cores,
            same workload and config.
N>1 (torchrun): every rank runs its own replica of the case (weak scaling);
timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import glob
import hashlib
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
L2_BYTES = 126 * 1024 * 1024
# algorithmic FP64 words per point-step: each globally dependent phase reads
# its inputs once and writes its outputs once.  Laminar: RHS 20, LU-SGS L 25,
# U 25, GS-L 30, GS-U 30, update + residual 15 = 145 (1,160 B).  The SA
# model adds qke/vist to the RHS, its own RHS, two scalar sweeps, the update
# and the wall distance: 195 words (1,560 B).
WORDS = {"laminar": 145, "sa": 195}
PHASE_WORDS = {"sweep_lusgs_l": 25, "sweep_lusgs_u": 25, "sweep_gs_pr_l": 30, "sweep_gs_pr_u": 30}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--case", default="channel")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-tune", action="store_true", help="run the default launch shapes (no autotuner)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the mixed-precision and 64-case batch measurements")
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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


def sources_digest():
    """SHA-256 over the CUDA sources, to tie a DRAM-traffic capture to the
    kernels it was taken from."""
    h = hashlib.sha256()
    for p in sorted(glob.glob(os.path.join(ROOT, "wcns_b200", "csrc", "*"))):
        with open(p, "rb") as f:
            h.update(os.path.basename(p).encode())
            h.update(f.read())
    return h.hexdigest()[:16]


def load_step_traffic(case_name, npoints):
    """DRAM bytes (read + write) of one time step, from the ncu summary of
    this workload under profiles/ (per point-step, scaled by the points).
    The summary records the digest of the CUDA sources it was captured with;
    when the sources have changed since, the figure is stale and None is
    returned with the reason."""
    path = os.path.join(ROOT, "profiles", f"{case_name}_step_dram.md")
    per, digest = None, None
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_point_step:"):
                per = float(line.split(":")[1])
            if line.startswith("sources_digest:"):
                digest = line.split(":")[1].strip()
    except OSError:
        return None, f"no capture summary {os.path.relpath(path, ROOT)}"
    if per is None:
        return None, "capture summary without a per-point figure"
    src = os.path.relpath(path, ROOT)
    if digest != sources_digest():
        return None, f"{src} was captured from other kernel sources (digest {digest})"
    return int(per * npoints), f"{src} (ncu dram__bytes_read.sum + dram__bytes_write.sum over one step's launches)"


def make_case(name):
    from wcns_b200 import cases
    return cases.CASES[name]()


def sa_prepare(obj, case):
    """Set up the SA model on a CUDA context when the workload has it (the
    reference's nlamtur=1, nameturb='SA')."""
    if case.sa:
        obj.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])


def sa_prepare_oracle(o, case):
    """The same on the oracle, whose brute-force wall distance would take
    minutes on the full channel: the distance comes from a k-d tree of the
    wall points instead (set-up work, outside every timed region)."""
    if not case.sa:
        return
    import numpy as np
    from scipy.spatial import cKDTree
    o.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"], distance=False)
    wall = []
    for r in case.regions:
        if int(r[7]) not in (2, 20, 21):
            continue
        x, y, z = case.xyz[int(r[0]) - 1]
        lo = [min(abs(r[1 + 2 * d]), abs(r[2 + 2 * d])) - 1 for d in range(3)]
        hi = [max(abs(r[1 + 2 * d]), abs(r[2 + 2 * d])) for d in range(3)]
        sl = (slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
        wall.append(np.stack([x[sl].ravel(), y[sl].ravel(), z[sl].ravel()], axis=1))
    if not wall:
        return
    tree = cKDTree(np.concatenate(wall))
    for nb, (x, y, z) in enumerate(case.xyz, start=1):
        ni, nj, nk = case.dims[nb - 1]
        d, _ = tree.query(np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1))
        full = np.zeros((nk + 6, nj + 6, ni + 6))
        full[3:3 + nk, 3:3 + nj, 3:3 + ni] = d.reshape(nk, nj, ni) + 1.0e-38
        o.set("dist", nb, full)


def config_of(case, world):
    resident = case_resident_bytes(case)
    return {"workload": f"{case.name}: {case.description}", "points": case.npoints, "blocks": case.nblocks,
            "nscheme": case.params.nscheme, "nflux": case.params.nflux, "nvis": case.params.nvis,
            "turbulence": "SA" if case.sa else "none", "mach": case.params.moo, "reynolds": case.params.reynolds,
            "l2": ("inputs larger than L2: %.1f GB of fields resident, steps back to back" % (resident / 1e9))
            if resident > 4 * L2_BYTES else "256 MiB L2 flush between timed steps",
            "parallelism": f"replicas x{world}"}


def case_resident_bytes(case):
    """Device bytes the step touches: the field pool (48 doubles per ghosted
    point), the sweep arrays and the SA fields."""
    ghosted = sum((a + 6) * (b + 6) * (c + 6) for a, b, c in case.dims)
    plane = sum((a + b + c - 2) * b * c for a, b, c in case.dims)
    return 8 * (48 * ghosted + 99 * plane + (8 * ghosted if case.sa else 0))


def cpu_reference_rate(case, steps, threads=None, target_s=None, max_s=None):
    """Oracle (CPU restatement) throughput on full steps of `case` after one
    untimed step.  With `target_s` the number of steps is chosen from the
    untimed step so that the timed sample lasts about that long; `max_s`
    caps the sample of a fixed step count."""
    from oracle.pyoracle import Oracle
    o = Oracle(case, nthreads=threads or os.cpu_count())
    sa_prepare_oracle(o, case)
    t0 = time.perf_counter()
    o.step(1)
    one = time.perf_counter() - t0
    if target_s:
        steps = int(min(200, max(steps, round(target_s / max(one, 1e-3)))))
    if max_s:
        steps = int(max(1, min(steps, max_s // max(one, 1e-3))))
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
    # each timed step is one full step of the workload on all host cores;
    # the count is capped so that the sample stays within about 100 s
    rate, dt, n = cpu_reference_rate(case, max(1, args.steps), cores, max_s=100.0)
    line = {
        "metric": METRIC, "value": round(rate, 4), "unit": "Mcell-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * dt / n, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": config_of(case, world),
        "cpu_baseline": {"value": round(rate, 4), "unit": "Mcell-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{n} full steps of the workload after 1 untimed step ({dt:.1f} s; OpenMP over "
                                   f"blocks and lines; the oracle restatement, the Fortran cannot be built here)"},
        "e2e": {"value": round(rate, 4), "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def profile_phases(g, reps=3):
    """Median device ms of every phase over `reps` profiled steps."""
    runs = [g.profile_step() for _ in range(reps)]
    out = []
    for q, (name, _) in enumerate(runs[0]):
        out.append((name, statistics.median(r[q][1] for r in runs)))
    return out


def timed_steps(g, steps, stream, flush=None):
    """Device ms of `steps` graph replays on the context's stream (back to
    back, or one by one after an L2 flush when `flush` is given)."""
    import torch
    torch.cuda.synchronize()
    if flush is None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step_async(steps)
        e1.record(stream)
        g.sync()
        return e0.elapsed_time(e1)
    evs = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
        g.step_async(1)
        b.record(stream)
        evs.append((a, b))
    g.sync()
    return sum(a.elapsed_time(b) for a, b in evs)


def rel_l2(a_ctx, b_ctx, names, dims, blocks_a=None, blocks_b=None):
    """Relative L2 (over the interior points) of every field of `names`:
    context a against context b, block lists matched in order."""
    import numpy as np
    ba = blocks_a or list(range(1, len(dims) + 1))
    bb = blocks_b or ba
    out = {}
    for name in names:
        num = den = 0.0
        for x, y in zip(ba, bb):
            ni, nj, nk = dims[y - 1]
            a = a_ctx.get(name, x)[3:3 + nk, 3:3 + nj, 3:3 + ni]
            b = b_ctx.get(name, y)[3:3 + nk, 3:3 + nj, 3:3 + ni]
            num += float(np.sum((a - b) ** 2))
            den += float(np.sum(b * b))
        out[name] = float((num / den) ** 0.5) if den > 0 else float(num ** 0.5)
    return out


def measure_mixed(case, value64, steps, warmup, tune=True):
    """The same workload with the mixed-precision residual: Mcell-steps/s,
    speed-up over the FP64 line and, after `warmup + steps` steps from the
    same start, the error of every variable and wall-force coefficient
    against a fresh FP64 context (the FP64 path equals the oracle to 1e-12)."""
    import torch
    from wcns_b200.solver import Wcns
    from wcns_b200 import autotune
    g = Wcns(case)
    sa_prepare(g, case)
    g.set_precision(32)
    shape = autotune.tuned(g)["shape"] if tune else g.shape
    stream = torch.cuda.ExternalStream(g.stream)
    g.step(warmup, history=False)
    ms = timed_steps(g, steps, stream)
    value = case.npoints * steps / (ms / 1e3) / 1e6
    ref = Wcns(case)
    sa_prepare(ref, case)
    ref.step(warmup + steps, history=False)
    names = ["r", "u", "v", "w", "p"] + (["qke"] if case.sa else [])
    err = rel_l2(g, ref, names, case.dims)
    fg, fr = g.force(), ref.force()
    g.close()
    ref.close()
    return {"value": round(value, 4), "unit": METRIC, "ms_per_step": round(ms / steps, 4),
            "speedup_vs_fp64": round(value / value64, 4), "shape": shape,
            "dtype": "f32 residual arithmetic; f64 metrics, IS denominators, dq sum, SA, LU-SGS, update",
            "after_steps": warmup + steps,
            "rel_l2_vs_fp64": {k: float(f"{v:.3e}") for k, v in err.items()},
            "force_rel_err_vs_fp64": force_errors(fg, fr)}


def force_errors(f, ref):
    """Errors of the wall-force coefficients cfx, cfy: each relative to its
    own value, and relative to the largest of |cfx|, |cfy|, |cfz| (a
    coefficient that is the small net of two walls' forces has no scale of
    its own)."""
    big = max(abs(ref[k]) for k in ("cfx", "cfy", "cfz"))
    out = {}
    for k in ("cfx", "cfy"):
        d = abs(f[k] - ref[k])
        out[k] = float(f"{d / max(abs(ref[k]), 1e-300):.3e}")
        out[k + "_vs_largest"] = float(f"{d / max(big, 1e-300):.3e}")
    out["values"] = {k: float(f"{ref[k]:.6e}") for k in ("cfx", "cfy")}
    return out


def measure_batch(steps, warmup, ncases=64, tune=True):
    """C4's batch: 64 independent small SA bump cases (block sizes 17^3 ..
    49x33x17, Mach U[0.3,0.8], bump U[0.02,0.08], seed 0).  Three forms, each
    `steps` steps after `warmup`, device-timed: every case on its own FP64
    context one after another (the plain per-case path), all cases in one
    FP64 context, and all cases in one context with the mixed-precision
    residual; then the errors of the mixed batch against the plain per-case
    runs (per-variable relative L2, the worst case's wall-force error)."""
    import torch
    from wcns_b200 import autotune, cases
    from wcns_b200.solver import Wcns
    b = cases.batch_case(ncases=ncases, seed=0)
    npts = b.npoints
    members = [cases.batch_member(b, q) for q in range(ncases)]
    sep_ms, singles = 0.0, []
    for m in members:
        h = Wcns(m)
        sa_prepare(h, m)
        if tune:
            autotune.tuned(h)
        h.step(warmup, history=False)
        sep_ms += timed_steps(h, steps, torch.cuda.ExternalStream(h.stream))
        singles.append(h)
    res = {"cases": ncases, "points": npts, "steps": steps,
           "fp64_separate": {"value": round(npts * steps / (sep_ms / 1e3) / 1e6, 4), "ms_per_step": round(sep_ms / steps, 4),
                      "note": "every case on its own context, one after another" + (", each autotuned" if tune else "")}}
    batched = {}
    for bits in (64, 32):
        g = Wcns(b)
        sa_prepare(g, b)
        g.set_precision(bits)
        if tune:
            autotune.tuned(g)
        g.step(warmup, history=False)
        ms = timed_steps(g, steps, torch.cuda.ExternalStream(g.stream))
        res[f"fp{bits}_batched"] = {"value": round(npts * steps / (ms / 1e3) / 1e6, 4), "ms_per_step": round(ms / steps, 4),
                                    "shape": g.shape}
        batched[bits] = g
    g = batched[32]
    names = ["r", "u", "v", "w", "p", "qke"]
    num = {k: 0.0 for k in names}
    den = {k: 0.0 for k in names}
    worst = {"cfx": 0.0, "cfy": 0.0, "cfx_vs_largest": 0.0, "cfy_vs_largest": 0.0}
    for q, h in enumerate(singles):
        nb0, _ = b.groups[q]
        e = rel_l2(g, h, names, members[q].dims, [nb0], [1])
        for k in names:  # pool the squared norms over the cases
            import numpy as np
            ni, nj, nk = members[q].dims[0]
            bref = h.get(k, 1)[3:3 + nk, 3:3 + nj, 3:3 + ni]
            d2 = float(np.sum(bref * bref))
            num[k] += (e[k] ** 2) * d2
            den[k] += d2
        fe = force_errors(g.force_blocks(nb0, nb0), h.force())
        for k in worst:
            worst[k] = max(worst[k], fe[k])
    for h in singles:
        h.close()
    for g in batched.values():
        g.close()
    sep = res["fp64_separate"]["value"]
    res["speedup_fp32_batched_vs_fp64_separate"] = round(res["fp32_batched"]["value"] / sep, 3)
    res["speedup_fp32_batched_vs_fp64_batched"] = round(res["fp32_batched"]["value"] / res["fp64_batched"]["value"], 3)
    res["fp32_batched_rel_l2_vs_fp64_separate"] = {k: float(f"{(num[k] / den[k]) ** 0.5:.3e}") for k in names}
    res["fp32_batched_worst_case_force_rel_err"] = {k: float(f"{v:.3e}") for k, v in worst.items()}
    return res


def run_b200(args, rank, world):
    import numpy as np
    import torch

    from wcns_b200 import autotune
    from wcns_b200.solver import Wcns
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    case = make_case(args.case)
    g = Wcns(case)
    sa_prepare(g, case)
    tune = autotune.tuned(g) if not args.no_tune else {"shape": g.shape, "source": "default"}
    stream = torch.cuda.ExternalStream(g.stream)
    big = case_resident_bytes(case) > 4 * L2_BYTES
    flush = None if big else torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    # warm-up
    g.step(args.warmup, history=False)
    dist_barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    if big:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step_async(args.steps)
        e1.record(stream)
        g.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    else:
        evs = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            g.step_async(1)
            b.record(stream)
            evs.append((a, b))
        g.sync()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
    clk = clocks.stop()
    dist_barrier(world)
    ms = dist_max(ms, world)
    total_points = case.npoints * world
    value = total_points * args.steps / (ms / 1e3) / 1e6
    step_ms = ms / args.steps

    # Roofline of the step program: one graph replay = one step of the whole
    # path.  Algorithmic bytes = the compulsory traffic of one point-step x
    # points; duration = the CUDA-event time per step above.
    peak, peak_kind = load_peak()
    words = WORDS["sa" if case.sa else "laminar"]
    step_bytes = case.npoints * words * 8
    achieved = step_bytes / (step_ms / 1e3) / 1e9
    traffic, traffic_src = load_step_traffic(case.name, case.npoints)

    # per-phase device times (one extra profiled step each, outside the timed region)
    phases = profile_phases(g)
    tot = sum(t for _, t in phases)
    ph = []
    for name, t in phases:
        e = {"phase": name, "ms": round(t, 4), "share": round(t / tot, 4) if tot else None}
        if name in PHASE_WORDS and t > 0:
            gbs = case.npoints * PHASE_WORDS[name] * 8 / (t / 1e3) / 1e9
            e.update(gbs=round(gbs, 1), frac=round(gbs / peak, 4))
        ph.append(e)
    dom = max(ph, key=lambda e: e["ms"])
    sweeps = [e for e in ph if e["phase"].startswith("sweep_")]

    # end-to-end through the C ABI with pinned host buffers: interior state in
    # and out in the flow-file layout
    names = ["r", "u", "v", "w", "p"] + (["qke"] if case.sa else [])
    pin = [[torch.empty((nk, nj, ni), dtype=torch.float64, pin_memory=True).numpy() for _ in names]
           for ni, nj, nk in case.dims]
    g.get_interior(names, pin)
    outs = [[torch.empty((nk, nj, ni), dtype=torch.float64, pin_memory=True).numpy() for _ in names]
            for ni, nj, nk in case.dims]
    h2d = sum(a.size * 8 for arrs in pin for a in arrs)
    d2h = sum(a.size * 8 for arrs in outs for a in arrs) + 8 * (2 * case.nblocks + 1)
    dist_barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        g.set_interior(names, pin)
        g.step(1, history=False)
        g.get_interior(names, outs)
        g.residual_curve()
    e2e_s = time.perf_counter() - t0
    e2e_s = dist_max(e2e_s, world)
    e2e = total_points * args.e2e_steps / e2e_s / 1e6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, dt, n = cpu_reference_rate(case, 3, os.cpu_count(), target_s=15.0)
            cpu = {"value": round(rate, 4), "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"{n} full steps of the workload after 1 untimed step ({dt:.1f} s, OpenMP)"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Mcell-steps/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {e}"}
    sweep_mode, launches = g.sweep_mode(), g.launches_per_step()
    g.close()
    mixed = batch = None
    if rank == 0 and world == 1 and not args.no_extra:
        mixed = measure_mixed(case, value, args.steps, args.warmup, not args.no_tune)
        batch = measure_batch(args.steps, args.warmup, tune=not args.no_tune)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "Mcell-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": config_of(case, world),
            "e2e": {"value": round(e2e, 4), "unit": "Mcell-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "roofline": {"bound": "hbm", "kernel": "one time step (CUDA graph of the whole path)",
                         "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 5), "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": int(step_bytes), "bytes_per_point_step": words * 8,
                         "launch_ms": round(step_ms, 4), "traffic": traffic, "traffic_source": traffic_src,
                         "dominant_phase": dom["phase"],
                         "sweeps": {"share": round(sum(e["share"] for e in sweeps), 4),
                                    "ms": round(sum(e["ms"] for e in sweeps), 4)}},
            "phases": ph,
            "sweep_mode": sweep_mode,
            "autotune": tune,
            "gpu_launches": launches * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        if mixed is not None:
            line["mixed_precision"] = mixed
            line["batch64"] = batch
        print(json.dumps(line), flush=True)
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
