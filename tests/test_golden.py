"""Committed golden fixtures (tests/golden/, made by make_golden.py from the
oracle on seeded cases): the oracle must reproduce them (CPU), and so must
the CUDA path through the C ABI (GPU) within the multi-step tolerance of the
parity tests.  The reference itself cannot run here, so these pin the
oracle's behaviour over time, not its agreement with the Fortran."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import GOLDEN, SA_GOLDEN, sa_prepare, summarize, summarize_sa

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_ORACLE = 1e-12
TOL_GPU = 1e-10


def load(name):
    with np.load(os.path.join(HERE, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def check(got, ref, tol):
    """Relative errors; velocity components are measured against the scale
    of the u component of the same block and quantity (a component that is
    zero in the free stream only carries round-off)."""
    assert set(got) | {"nsteps"} == set(ref)
    bad = {}
    for k, v in got.items():
        scale = np.abs(ref[k]).max()
        if k != "rms":
            blk, var, kind = k.split("_", 2)
            if var in ("v", "w"):
                scale = max(scale, np.abs(ref[f"{blk}_u_{kind}"]).max())
            if kind == "pts":
                scale = max(scale, np.abs(ref[k]).mean())
        e = np.abs(np.asarray(v) - ref[k]).max() / scale if scale > 0 else np.abs(v).max()
        if e > tol:
            bad[k] = e
    assert not bad, bad


@pytest.mark.parametrize("name", list(GOLDEN))
def test_oracle_reproduces_golden(oracle_lib, name):
    make, nsteps = GOLDEN[name]
    case = make()
    o = oracle_lib.Oracle(case)
    hist = o.step(nsteps)
    check(summarize(o.get, case, hist), load(name), TOL_ORACLE)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(GOLDEN))
def test_cuda_path_reproduces_golden(name):
    from wcns_b200.solver import Wcns
    make, nsteps = GOLDEN[name]
    case = make()
    g = Wcns(case)
    hist = g.step(nsteps)
    check(summarize(g.get, case, hist), load(name), TOL_GPU)
    g.close()


@pytest.mark.parametrize("name", list(SA_GOLDEN))
def test_oracle_reproduces_sa_golden(oracle_lib, name):
    make, nsteps, tt, km = SA_GOLDEN[name]
    case = make()
    o = oracle_lib.Oracle(case)
    sa_prepare(o, case, tt, km)
    hist = o.step(nsteps)
    check(summarize_sa(o.get, case, hist), load(name), TOL_ORACLE)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SA_GOLDEN))
def test_cuda_path_reproduces_sa_golden(name):
    from wcns_b200.solver import Wcns
    make, nsteps, tt, km = SA_GOLDEN[name]
    case = make()
    g = Wcns(case)
    sa_prepare(g, case, tt, km)
    hist = g.step(nsteps)
    check(summarize_sa(g.get, case, hist), load(name), TOL_GPU)
    g.close()
