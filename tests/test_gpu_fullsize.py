"""GPU parity at the benchmark configurations' full sizes.

C1: the isentropic vortex on one 65x33x17 block (nscheme 4, Steger-Warming),
all 100 steps of the configuration.  C2: the 8-block laminar plate with its
228,888 points (nscheme 41, Roe), 20 steps.  The CUDA path (CUDA graph of
whole steps) against the oracle on the same seeded inputs: residual history
and primitive fields after the last step, 1e-10 relative (velocity
components relative to the flow speed)."""
import numpy as np
import pytest

from tests.helpers import compare_prim_scaled
from wcns_b200 import cases

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _run(case, n):
    from oracle.pyoracle import Oracle
    from wcns_b200.solver import Wcns
    g, o = Wcns(case), Oracle(case)
    hg, ho = g.step(n), o.step(n)
    return g, o, hg, ho


def test_c1_vortex_full_100_steps():
    case = cases.vortex_case()
    assert case.npoints == 36_465
    g, o, hg, ho = _run(case, 100)
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= TOL
    errs = compare_prim_scaled(g, o)
    assert max(errs.values()) <= TOL, errs


def test_c2_plate_full_20_steps():
    case = cases.plate_case()
    assert case.npoints == 228_888
    g, o, hg, ho = _run(case, 20)
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= TOL
    errs = compare_prim_scaled(g, o)
    assert max(errs.values()) <= TOL, errs
