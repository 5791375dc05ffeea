"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Both sides start from the same seeded inputs.  Phase-by-phase comparisons
must agree to FP64 round-off: the kernels restate the reference operation
sequence with fused multiply-add disabled, so most fields are bitwise equal;
the far-field boundary uses pow(), where CUDA's and glibc's results may differ
in the last bit, so the bar is a relative error of 1e-12 per field.
"""
import numpy as np
import pytest

from tests.helpers import compare_fields, compare_prim_scaled, interior, perturbed, rel_err, supersonic_box_case, with_params
from wcns_b200 import cases

pytestmark = pytest.mark.gpu

TOL_PHASE = 1e-12
TOL_STEPS = 1e-10
PRIM = ["r", "u", "v", "w", "p"]
METRICS = ["kcx", "kcy", "kcz", "etx", "ety", "etz", "ctx", "cty", "ctz", "vol"]
DQ = ["dq1", "dq2", "dq3", "dq4", "dq5"]


def make_pair(case):
    from oracle.pyoracle import Oracle
    from wcns_b200.solver import Wcns
    return Wcns(case), Oracle(case)


CASES = {
    "vortex_sw_4": lambda: cases.vortex_case(ni=33, nj=17, nk=9, nscheme=4, nflux=1),
    "vortex_roe_41": lambda: cases.vortex_case(ni=33, nj=17, nk=9, nscheme=41, nflux=3),
    "plate_small": lambda: cases.small_plate_case(),
    "plate_small_nscheme4_sw": lambda: cases.small_plate_case(nscheme=4, nflux=1),
    # boundary-condition coverage: adiabatic wall, inviscid wall, 2-D symmetry
    # (nk <= 4), supersonic inflow/outflow
    "plate_small_adiabatic": lambda: with_params(cases.small_plate_case(), twall=-1.0),
    "plate_small_euler_wall": lambda: perturbed(with_params(cases.small_plate_case(nscheme=4, nflux=1), nvis=0)),
    "plate_small_sym2d": lambda: cases.small_plate_case(nk=4),
    "supersonic_box_roe41": lambda: supersonic_box_case(),
    "supersonic_box_sw4": lambda: supersonic_box_case(nscheme=4, nflux=1),
    # Van Leer flux (nflux 2): subsonic vortex and plate, supersonic box
    "vortex_vl_4": lambda: cases.vortex_case(ni=33, nj=17, nk=9, nscheme=4, nflux=2),
    "plate_small_vl41": lambda: cases.small_plate_case(nflux=2),
    "supersonic_box_vl41": lambda: supersonic_box_case(nscheme=41, nflux=2),
    # nscheme 42: the 41 boundary sections with second-order end states
    "vortex_roe_42": lambda: cases.vortex_case(ni=33, nj=17, nk=9, nscheme=42, nflux=3),
    "plate_small_roe42": lambda: cases.small_plate_case(nscheme=42),
    "supersonic_box_sw42": lambda: supersonic_box_case(nscheme=42, nflux=1),
}


@pytest.mark.parametrize("name", list(CASES))
def test_metrics_bitwise(name):
    g, o = make_pair(CASES[name]())
    errs = compare_fields(g, o, METRICS)
    assert max(errs.values()) == 0.0, errs


@pytest.mark.parametrize("name", list(CASES))
def test_phase_by_phase(name):
    case = CASES[name]()
    g, o = make_pair(case)
    report = {}

    def cmp(tag, names, region="interior", tol=TOL_PHASE):
        e = compare_fields(g, o, names, region=region)
        report[tag] = e
        assert max(e.values()) <= tol, (tag, e)

    for step in range(2):
        g.boundary_all(); o.phase("boundary_all")
        cmp(f"{step}:bc", PRIM, region="all")
        g.initial_q_dq_c_t(); o.phase("initial_q_dq_c_t")
        if case.params.nvis == 1:
            cmp(f"{step}:t", ["t"], region="all")
        g.timestep_tgh(); o.phase("timestep")
        cmp(f"{step}:dt", ["dtdt", "sra", "srb", "src", "srva", "srvb", "srvc"])
        if case.params.nvis == 1:
            g.r_h_s_vis(); o.phase("rhs_vis")
            cmp(f"{step}:vis", DQ)
            g.communicate_dq_npp(); o.phase("communicate_dq")
            cmp(f"{step}:cdq1", DQ)
        g.r_h_s_invis(); o.phase("rhs_invis")
        cmp(f"{step}:inv", DQ)
        g.communicate_dq_npp(); o.phase("communicate_dq")
        cmp(f"{step}:cdq2", DQ)
        g.l_h_s_tgh(); o.phase("lhs")
        cmp(f"{step}:lhs_dq", DQ)
        cmp(f"{step}:lhs_prim", PRIM)
        g.communicate_pv_npp(); o.phase("communicate_pv")
        cmp(f"{step}:cpv", PRIM + (["t"] if case.params.nvis == 1 else []))
        res_g = g.residual_curve()
        res_o = o.residual()
        assert rel_err(res_g[0], res_o[0]) <= 1e-12
        assert rel_err(res_g[1], res_o[1]) <= 1e-12
        assert abs(res_g[2] - res_o[2]) <= 1e-12 * abs(res_o[2])
    print(name, {k: max(v.values()) for k, v in report.items()})


@pytest.mark.parametrize("name", list(CASES))
def test_multistep_graph(name):
    case = CASES[name]()
    g, o = make_pair(case)
    n = 20
    hg = g.step(n)
    ho = o.step(n)
    assert np.max(np.abs(hg - ho) / np.abs(ho)) <= TOL_STEPS, (hg, ho)
    errs = compare_prim_scaled(g, o)
    print(name, "20 steps", errs, "rms", hg[-1])
    assert max(errs.values()) <= TOL_STEPS, errs


def test_graph_step_equals_phase_calls():
    case = cases.small_plate_case()
    from wcns_b200.solver import Wcns
    a, b = Wcns(case), Wcns(case)
    a.step(3)
    for _ in range(3):
        b.boundary_all(); b.initial_q_dq_c_t(); b.timestep_tgh(); b.r_h_s_vis(); b.communicate_dq_npp()
        b.r_h_s_invis(); b.communicate_dq_npp(); b.l_h_s_tgh(); b.communicate_pv_npp()
    for nb in range(1, case.nblocks + 1):
        for f in PRIM:
            assert np.array_equal(interior(a.get(f, nb), case.dims[nb - 1]), interior(b.get(f, nb), case.dims[nb - 1]))


FORCE_REF = dict(sref=2.0, lfref=0.5, xref=0.25, yref=0.0, zref=0.01, nwholefield=1)


def test_wall_forces_match_oracle():
    """force_dif/getforce on the device against the oracle after two steps of
    the laminar plate: pressure and viscous stress, summed in the reference's
    loop order (relative to the largest coefficient)."""
    g, o = make_pair(cases.small_plate_case())
    g.step(2)
    o.step(2)
    fg, fo = g.force(**FORCE_REF), o.force(**FORCE_REF)
    scale = max(abs(fo[k]) for k in ("cfx", "cfy", "cfz"))
    for k in ("cfx", "cfy", "cfz", "cmx", "cmy", "cmz", "cl", "cd"):
        assert abs(fg[k] - fo[k]) <= TOL_PHASE * max(scale, abs(fo[k])), (k, fg[k], fo[k])
    assert fg["xcp"] == pytest.approx(fo["xcp"], rel=1e-10)


def test_no_walls_no_force():
    g = make_pair(CASES["vortex_sw_4"]())[0]
    f = g.force()
    assert all(v == 0.0 for v in f.values())


def test_get_prim_equals_get_field():
    """wcns_get_prim returns, block by block, exactly what wcns_get_field
    returns for r, u, v, w, p, T; with five arrays it leaves T alone."""
    g = make_pair(cases.small_plate_case())[0]
    g.step(2)
    for nb in range(1, len(g.dims) + 1):
        got = g.get_prim(nb)
        for a, name in zip(got, ("r", "u", "v", "w", "p", "t")):
            assert np.array_equal(a, g.get(name, nb)), (nb, name)
        five = [np.empty_like(a) for a in got[:5]]
        g.get_prim(nb, out=five)
        for a, b in zip(five, got[:5]):
            assert np.array_equal(a, b)


def test_all_block_state_transfer():
    """wcns_set_prim_all / wcns_get_prim_all move every block's state with one
    synchronisation and agree exactly with the per-block calls."""
    case = cases.small_plate_case()
    from wcns_b200.solver import Wcns
    a, b = Wcns(case), Wcns(case)
    a.step(2)
    states = [a.get_prim(nb) for nb in range(1, case.nblocks + 1)]
    b.set_prim_all(states)
    outs = [[np.zeros_like(x) for x in st[:5]] for st in states]
    b.get_prim_all(outs)
    for st, out in zip(states, outs):
        for x, y in zip(st[:5], out):
            assert np.array_equal(x, y)
    a.step(3)
    b.step(3)
    for nb in range(1, case.nblocks + 1):
        for x, y in zip(a.get_prim(nb), b.get_prim(nb)):
            assert np.array_equal(x, y)


def test_get_flow_is_the_interior():
    """wcns_get_flow returns each block's interior points in the flow-file
    layout, exactly the interior of what wcns_get_prim returns."""
    case = cases.small_plate_case()
    from wcns_b200.solver import Wcns
    g = Wcns(case)
    g.step(2)
    flow = g.get_flow()
    for nb in range(1, case.nblocks + 1):
        full = g.get_prim(nb)
        for x, y in zip(full, flow[nb - 1]):
            assert np.array_equal(interior(x, case.dims[nb - 1]), y)
    five = [[np.zeros_like(a) for a in blk[:5]] for blk in flow]
    g.get_flow(five)
    for a, b in zip(five, flow):
        for x, y in zip(a, b[:5]):
            assert np.array_equal(x, y)


# the sweeps as one launch per hyperplane (the path of blocks too large for
# the clustered sweep kernel), asked for on cases that would use the kernel
PLANE_CASES = ["vortex_roe_41", "plate_small", "plate_small_euler_wall", "supersonic_box_sw4"]


@pytest.mark.parametrize("mode", ["plane", "wide", "wide_narrow"])
@pytest.mark.parametrize("name", PLANE_CASES)
def test_sweep_variants_match_oracle(name, mode, monkeypatch):
    """The sweeps as one launch per hyperplane, and as wide cooperative
    sweeps: with the default chunking and with chunks of one j-row each
    (WCNS_WIDE_MIN_COLS=1 on these small blocks), where every j contribution
    crosses a ring between CTAs."""
    from oracle.pyoracle import Oracle
    from wcns_b200.solver import FLAG_SWEEP_BY_PLANE, FLAG_SWEEP_WIDE, Wcns
    if mode == "wide_narrow":
        monkeypatch.setenv("WCNS_WIDE_MIN_COLS", "1")
    case = CASES[name]()
    g, o = Wcns(case, flags=FLAG_SWEEP_BY_PLANE if mode == "plane" else FLAG_SWEEP_WIDE), Oracle(case)
    for gp, op in [("boundary_all", "boundary_all"), ("initial_q_dq_c_t", "initial_q_dq_c_t"),
                   ("timestep_tgh", "timestep")] + ([("r_h_s_vis", "rhs_vis"), ("communicate_dq_npp", "communicate_dq")]
                                                    if case.params.nvis else []) + \
                  [("r_h_s_invis", "rhs_invis"), ("communicate_dq_npp", "communicate_dq"), ("l_h_s_tgh", "lhs")]:
        getattr(g, gp)()
        o.phase(op)
    e = compare_fields(g, o, DQ + PRIM)
    assert max(e.values()) <= TOL_PHASE, e
    g.communicate_pv_npp(); o.phase("communicate_pv")
    hg, ho = g.step(5), o.step(5)
    np.testing.assert_allclose(hg, ho, rtol=1e-12, atol=0)
    e = compare_prim_scaled(g, o)
    assert max(e.values()) <= 1e-12, e
