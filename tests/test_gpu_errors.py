"""Error and fallback paths on the GPU, each set up from the host and none
of them faulting the device.

* update_limited's neighbour-average fallback (Sub2.f90:603-794): a point
  whose updated pressure reaches pmax_limit (1e3) is replaced by the mean of
  its six neighbours, the lower ones already updated and the upper ones not
  yet (the reference's loop order).  A few isolated high-pressure points
  (p = 1200) set with wcns_set_prim trigger it; the GPU result must equal
  the oracle's and that formula.
* the bad-point limit (more than ni*nj*nk/64 or 500 points, Sub2.f90:781-785)
  stops the reference; here wcns_lhs returns WCNS_ERR_UPDATE and a
  multi-step wcns_step stops after the failing step.
* the LU-SGS sweeps' bounded waits: wcns_selftest_timeout runs the same wait
  on an mbarrier that nothing completes, with a short limit; the call
  reports WCNS_ERR_CUDA and the context keeps working.
"""
import numpy as np
import pytest

from tests.helpers import compare_fields
from wcns_b200 import cases

pytestmark = pytest.mark.gpu

SPOTS = [(5, 4, 3), (12, 9, 5), (15, 6, 4)]  # (i, j, k) in block 1 (17 x 11 x 7)
BEFORE_LHS = [("boundary_all", "boundary_all"), ("initial_q_dq_c_t", "initial_q_dq_c_t"), ("timestep_tgh", "timestep"),
              ("r_h_s_vis", "rhs_vis"), ("communicate_dq_npp", "communicate_dq"), ("r_h_s_invis", "rhs_invis"),
              ("communicate_dq_npp", "communicate_dq")]


def spiked_plate(spots, value=1200.0):
    case = cases.small_plate_case()
    p = case.prim[0][4]
    for (i, j, k) in spots:
        p[k + 2, j + 2, i + 2] = value
    return case


def _pair(case):
    from oracle.pyoracle import Oracle
    from wcns_b200.solver import Wcns
    return Wcns(case), Oracle(case)


def test_update_fallback_matches_oracle_and_formula():
    g, o = _pair(spiked_plate(SPOTS))
    for gp, op in BEFORE_LHS:
        getattr(g, gp)()
        o.phase(op)
    names = ("r", "u", "v", "w", "p")
    old = {n: g.get(n, 1) for n in names}
    g.l_h_s_tgh()
    o.phase("lhs")
    e = compare_fields(g, o, list(names))
    assert max(e.values()) <= 1e-12, e
    new = {n: g.get(n, 1) for n in names}
    for (i, j, k) in SPOTS:
        c = (k + 2, j + 2, i + 2)
        lower = [(k + 2, j + 2, i + 1), (k + 2, j + 1, i + 2), (k + 1, j + 2, i + 2)]
        upper = [(k + 3, j + 2, i + 2), (k + 2, j + 3, i + 2), (k + 2, j + 2, i + 3)]
        for n in names:
            acc = 0.0
            for idx in lower:
                acc = acc + new[n][idx]
            for idx in upper:  # in the reference's order: k+1, j+1, i+1
                acc = acc + old[n][idx]
            assert new[n][c] == acc / 6.0, (i, j, k, n)
        assert new["p"][c] < 1.0e3


def test_bad_point_limit_stops_phase_and_step():
    # a 5 x 3 x 3 high-pressure region: 45 bad points > 17*11*7/64
    region = [(i, j, k) for i in range(5, 10) for j in range(4, 7) for k in range(2, 5)]
    from wcns_b200.solver import WcnsError
    g, o = _pair(spiked_plate(region))
    for gp, op in BEFORE_LHS:
        getattr(g, gp)()
        o.phase(op)
    with pytest.raises(WcnsError) as ei:
        g.l_h_s_tgh()
    assert ei.value.code == 3 and "non-physical" in str(ei.value)
    with pytest.raises(RuntimeError):
        o.phase("lhs")
    # a multi-step call stops after the failing first step
    g2, o2 = _pair(spiked_plate(region))
    hist = np.zeros(5)
    from wcns_b200 import _lib
    rc = _lib.load().wcns_step(g2.h, 5, hist.ctypes.data)
    assert rc == 3
    assert "step 1 of 5" in _lib.last_error()
    assert np.all(hist[1:] == 0.0) and hist[0] != 0.0
    with pytest.raises(RuntimeError):
        o2.step(5)


def test_sweep_wait_timeout_is_reported_and_context_survives():
    from wcns_b200.solver import WcnsError
    case = cases.small_plate_case()
    g, o = _pair(case)
    with pytest.raises(WcnsError) as ei:
        g.selftest_timeout(1000)
    assert ei.value.code == 4 and "bounded wait" in str(ei.value)
    # the error slots were cleared by the report; the next steps run normally
    hg, ho = g.step(2), o.step(2)
    np.testing.assert_allclose(hg, ho, rtol=1e-12, atol=0)
    e = compare_fields(g, o, ["r", "u", "v", "w", "p"])
    assert max(e.values()) <= 1e-12, e
