"""Mixed-precision residual (wcns_set_precision(ctx, 32)): FP32
interpolation, fluxes and viscous arithmetic; FP64 metrics, smoothness-
indicator denominators, dq accumulation, time step, SA model and LU-SGS.

The mixed form is not a restatement of the reference's operation order, so
it is measured against the FP64 path (which itself equals the oracle to
1e-12): its error is stated per quantity and bounded here.
  * one residual evaluation on the same state: dq relative to the case's
    largest |dq|;
  * whole steps on the reduced SA channel against the oracle: per-variable
    relative L2 of r, u, v, w, p, qke and the wall-force coefficients;
  * switching back to 64 restores the FP64 path bit for bit (the captured
    step graph is dropped with the precision)."""
import numpy as np
import pytest

from tests.helpers import interior, perturbed, supersonic_box_case
from wcns_b200 import cases

pytestmark = pytest.mark.gpu


def _case(name):
    if name == "vortex":
        return cases.vortex_case(ni=33, nj=17, nk=9, nsteps=5)
    if name == "plate":
        return perturbed(cases.small_plate_case())
    if name == "box41":
        return supersonic_box_case(nscheme=41)
    if name == "box42_vl":
        return supersonic_box_case(nscheme=42, nflux=2)
    if name == "channel":
        return cases.small_channel_case()
    raise KeyError(name)


def _ctx(case, bits):
    from wcns_b200.solver import Wcns
    g = Wcns(case)
    if case.sa:
        g.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    g.set_precision(bits)
    assert g.precision == bits
    return g


def _residual(g, case):
    g.boundary_all()
    g.initial_q_dq_c_t()
    g.timestep_tgh()
    if case.params.nvis == 1:
        g.r_h_s_vis()
    g.r_h_s_invis()
    return [[interior(g.get(f"dq{m}", nb), case.dims[nb - 1]) for m in range(1, 6)]
            for nb in range(1, case.nblocks + 1)]


@pytest.mark.parametrize("name", ["vortex", "plate", "box41", "box42_vl", "channel"])
def test_mixed_residual_one_evaluation(name):
    case = _case(name)
    a = _residual(_ctx(case, 64), case)
    b = _residual(_ctx(case, 32), case)
    # each component relative to its own largest |dq|; the three momentum
    # components relative to the largest of them (one can be zero by symmetry)
    amax = [max(float(np.max(np.abs(blk[m]))) for blk in a) for m in range(5)]
    scales = [amax[0], *([max(amax[1:4])] * 3), amax[4]]
    errs = []
    for m in range(5):
        diff = max(float(np.max(np.abs(x[m] - y[m]))) for x, y in zip(a, b))
        errs.append(diff / scales[m] if scales[m] > 0 else diff)
    print(f"{name}: dq error relative to max|dq| per component", " ".join(f"{e:.2e}" for e in errs))
    # measured on B200: <= 8e-6 (Van Leer, nscheme 42), <= 2.3e-6 elsewhere
    assert max(errs) < 5e-5, errs


def _rel_l2(g, o, name, dims):
    num = den = 0.0
    for nb in range(1, len(dims) + 1):
        a, b = interior(g.get(name, nb), dims[nb - 1]), interior(o.get(name, nb), dims[nb - 1])
        num += float(np.sum((a - b) ** 2))
        den += float(np.sum(b * b))
    return (num / den) ** 0.5 if den > 0 else num ** 0.5


def test_mixed_steps_error_table():
    """The reduced SA channel, 50 steps of the mixed form against the FP64
    oracle: relative L2 per variable and the wall-force coefficients."""
    from oracle.pyoracle import Oracle
    case = cases.small_channel_case()
    n = 50
    g = _ctx(case, 32)
    g.step(n, history=False)
    o = Oracle(case)
    o.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    for nb in range(1, case.nblocks + 1):  # the same wall distance (exact minimum on both)
        o.set("dist", nb, g.get("dist", nb))
    o.step(n)
    l2 = {name: _rel_l2(g, o, name, case.dims) for name in ("r", "u", "v", "w", "p", "qke")}
    fg, fo = g.force(), o.force()
    cf = {}
    for k in ("cfx", "cfy"):
        cf[k] = abs(fg[k] - fo[k]) / abs(fo[k])
    print("mixed, reduced SA channel, 50 steps: rel L2", {k: f"{v:.2e}" for k, v in l2.items()},
          "force", {k: f"{v:.2e}" for k, v in cf.items()})
    # measured on B200: r, u, p <= 7e-9, qke 7e-8, cfx 1.2e-8, cfy 6.5e-7
    # (cfy is the small net of the two walls' gauge-pressure forces)
    assert max(l2[k] for k in ("r", "u", "p")) < 1e-6, l2
    assert l2["qke"] < 1e-5, l2
    assert max(cf.values()) < 1e-5, cf


def test_precision_switch_back_is_fp64():
    """32 for two steps, then 64: the next steps are the FP64 path's, bit
    for bit (a laminar case: its state is the prim fields)."""
    case = cases.small_plate_case()
    a = _ctx(case, 32)
    a.step(2, history=False)
    prim = [a.get_prim(nb) for nb in range(1, case.nblocks + 1)]
    a.set_precision(64)
    ha = a.step(2)
    b = _ctx(case, 64)
    for nb in range(1, case.nblocks + 1):
        b.set_prim(nb, prim[nb - 1])
    hb = b.step(2)
    np.testing.assert_array_equal(ha, hb)
    for nb in range(1, case.nblocks + 1):
        for f in ("r", "u", "v", "w", "p"):
            np.testing.assert_array_equal(a.get(f, nb), b.get(f, nb))


def test_set_precision_rejects_other_values():
    from wcns_b200.solver import Wcns, WcnsError
    g = Wcns(cases.small_plate_case())
    with pytest.raises(WcnsError):
        g.set_precision(16)
    assert g.precision == 64
