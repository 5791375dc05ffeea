"""Runs a few whole steps of a seeded case, for profilers (ncu) to capture.

    python -m wcns_b200.profile_step --case channel --kw ni=129 nj=155 nk=43 bx=2 by=2 bz=1 \\
        --steps 2 [--wide] [--mixed] [--tune]

--case names a generator of wcns_b200.cases (channel, small_channel, plate,
small_plate, vortex, batch) and --kw passes its keyword arguments (integers
and floats).  The SA model is set up when the case
has one.  --wide sweeps with the wide cooperative kernels, --mixed runs the
mixed-precision residual, --tune applies the autotuned shape first.  Prints
the points, the sweep mode, the shape and the device ms per step (CUDA
events around the steps, which a profiler's replay inflates).
"""
from __future__ import annotations

import argparse
import json
import sys


def _value(v: str):
    for cast in (int, float):
        try:
            return cast(v)
        except ValueError:
            pass
    return v


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m wcns_b200.profile_step")
    ap.add_argument("--case", default="small_channel")
    ap.add_argument("--kw", nargs="*", default=[])
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--wide", action="store_true")
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--tune", action="store_true")
    a = ap.parse_args(argv)
    from . import autotune, cases
    from .solver import FLAG_SWEEP_WIDE, Wcns
    kw = {}
    for item in a.kw:
        k, _, v = item.partition("=")
        kw[k] = _value(v)
    case = cases.CASES[a.case](**kw)
    g = Wcns(case, flags=FLAG_SWEEP_WIDE if a.wide else 0)
    if case.sa:
        g.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    if a.mixed:
        g.set_precision(32)
    if a.tune:
        autotune.tuned(g, use_cache=False)
    import ctypes
    from . import _lib
    lib = _lib.load()
    g.step(a.steps, history=False)
    # device time of the steps, by CUDA events on the context's stream
    cudart = ctypes.CDLL("libcudart.so")
    ev = [ctypes.c_void_p(), ctypes.c_void_p()]
    for e in ev:
        cudart.cudaEventCreate(ctypes.byref(e))
    stream = ctypes.c_void_p(g.stream)
    cudart.cudaEventRecord(ev[0], stream)
    g.step_async(a.steps)
    cudart.cudaEventRecord(ev[1], stream)
    g.sync()
    ms = ctypes.c_float(0.0)
    cudart.cudaEventElapsedTime(ctypes.byref(ms), ev[0], ev[1])
    print(json.dumps({"case": a.case, "kw": kw, "points": case.npoints, "sweep_mode": g.sweep_mode(),
                      "shape": g.shape, "precision": g.precision, "ms_per_step": round(ms.value / a.steps, 4)}))
    del lib
    g.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
