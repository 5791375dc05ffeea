"""Generates the golden fixtures of tests/test_golden.py from the CPU oracle.

    python tests/golden/make_golden.py

The reference (Fortran + MPI) cannot be built or run in this environment and
ships no test vectors, so these fixtures pin the oracle's own output on
seeded synthetic cases: a regression pin for the oracle and a fixed target
for the CUDA path, not a pin against the reference.  Each fixture holds,
after `nsteps` full steps: the residual RMS of every step, per block and
variable the sum and the L2 norm of the interior primitive field, and the
values at 64 seeded interior points per block.
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


def main():
    from oracle.pyoracle import Oracle, build
    build()
    for name, (make, nsteps) in GOLDEN.items():
        case = make()
        o = Oracle(case)
        hist = o.step(nsteps)
        np.savez(os.path.join(HERE, name + ".npz"), nsteps=np.array([nsteps]), **summarize(o.get, case, hist))
        o.close()
        print("wrote", name)


if __name__ == "__main__":
    main()
