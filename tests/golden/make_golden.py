"""Generates the golden fixtures of tests/test_golden.py from the CPU oracle.

    python tests/golden/make_golden.py

The reference (Fortran + MPI) cannot be built or run in this environment and
ships no test vectors, so these fixtures pin the oracle's own output on
seeded synthetic cases: a regression pin for the oracle and a fixed target
for the CUDA path, not a pin against the reference.  Each fixture holds,
after `nsteps` full steps: the residual RMS of every step, per block and
variable the sum and the L2 norm of the interior primitive field, and the
values at 64 seeded interior points per block (for the SA runs also qke and
vist).  `python tests/golden/make_golden.py NAME ...` writes only the named
fixtures.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from wcns_b200 import cases  # noqa: E402

GOLDEN = {
    "small_plate_roe41_vis": (lambda: cases.small_plate_case(), 3),
    "vortex_sw4": (lambda: cases.vortex_case(ni=33, nj=17, nk=9, nscheme=4, nflux=1), 3),
    "vortex_roe41": (lambda: cases.vortex_case(ni=33, nj=17, nk=9, nscheme=41, nflux=3), 3),
}
PRIM = ("r", "u", "v", "w", "p")

# Spalart-Allmaras runs: the model set up (timedt_turb, kmaxlim) and a seeded
# non-uniform qke, then whole steps with the model coupled to the mean flow
# and its qke/vist boundary rules applied in boundary_all
SA_GOLDEN = {
    "small_plate_sa": (lambda: cases.small_plate_case(), 3, 1.0, 0.0),
    "small_channel_sa": (lambda: cases.small_channel_case(), 3, 10.0, 30000.0),
}


def sa_prepare(obj, case, timedt_turb, kmaxlim):
    """Set up the model on an oracle or a CUDA context and seed qke."""
    obj.sa_setup(timedt_turb, kmaxlim)
    rng = np.random.default_rng(21)
    for nb, (ni, nj, nk) in enumerate(case.dims, start=1):
        obj.set("qke", nb, 0.1 * (1.0 + 20.0 * rng.random((nk + 6, nj + 6, ni + 6))))


def sample_points(dims, nb, n=64):
    rng = np.random.default_rng(1000 + nb)
    ni, nj, nk = dims
    return np.stack([rng.integers(0, nk, n), rng.integers(0, nj, n), rng.integers(0, ni, n)], axis=1)


def summarize(get, case, hist):
    out = {"rms": np.asarray(hist, dtype=np.float64)}
    for nb, d in enumerate(case.dims, start=1):
        pts = sample_points(d, nb)
        for name in PRIM:
            a = cases.interior(get(name, nb), d)
            out[f"b{nb}_{name}_sum"] = np.array([a.sum()])
            out[f"b{nb}_{name}_l2"] = np.array([np.sqrt((a * a).sum())])
            out[f"b{nb}_{name}_pts"] = a[pts[:, 0], pts[:, 1], pts[:, 2]].copy()
    return out


def summarize_sa(get, case, hist):
    out = summarize(get, case, hist)
    for nb, d in enumerate(case.dims, start=1):
        pts = sample_points(d, nb)
        for name in ("qke", "vist"):
            a = cases.interior(get(name, nb), d)
            out[f"b{nb}_{name}_sum"] = np.array([a.sum()])
            out[f"b{nb}_{name}_l2"] = np.array([np.sqrt((a * a).sum())])
            out[f"b{nb}_{name}_pts"] = a[pts[:, 0], pts[:, 1], pts[:, 2]].copy()
    return out


def main(names=None):
    from oracle.pyoracle import Oracle, build
    build()
    for name, (make, nsteps, tt, km) in SA_GOLDEN.items():
        if names and name not in names:
            continue
        case = make()
        o = Oracle(case)
        sa_prepare(o, case, tt, km)
        hist = o.step(nsteps)
        np.savez(os.path.join(HERE, name + ".npz"), nsteps=np.array([nsteps]), **summarize_sa(o.get, case, hist))
        o.close()
        print("wrote", name)
    for name, (make, nsteps) in GOLDEN.items():
        if names and name not in names:
            continue
        case = make()
        o = Oracle(case)
        hist = o.step(nsteps)
        np.savez(os.path.join(HERE, name + ".npz"), nsteps=np.array([nsteps]), **summarize(o.get, case, hist))
        o.close()
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
