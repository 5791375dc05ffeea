"""Spalart-Allmaras model (turbulence -> differential_model_turbulence,
turblence.f90:15-103): oracle known-answer tests on the CPU and GPU parity
through the C ABI.

GPU and oracle evaluate pow() in the source term and in fv1 (CUDA's and
glibc's results may differ in the last bit), so qke and vist are compared
with a relative bar of 1e-12; the wall distance is an exact minimum and must
agree bitwise."""
import numpy as np
import pytest

from tests.helpers import compare_fields, interior, supersonic_box_case, with_params
from wcns_b200 import cases

TOL = 1e-12
MUOO = 0.1
CV13 = 7.1 ** 3.0


def wall_points(case):
    pts = []
    for nb, (x, y, z) in enumerate(case.xyz, start=1):
        for r in case.regions:
            if r[0] != nb or r[7] not in (2, 20, 21):
                continue
            lo = [min(abs(r[1 + 2 * d]), abs(r[2 + 2 * d])) for d in range(3)]
            hi = [max(abs(r[1 + 2 * d]), abs(r[2 + 2 * d])) for d in range(3)]
            sl = (slice(lo[2] - 1, hi[2]), slice(lo[1] - 1, hi[1]), slice(lo[0] - 1, hi[0]))
            pts.append(np.stack([x[sl].ravel(), y[sl].ravel(), z[sl].ravel()], axis=1))
    return np.concatenate(pts) if pts else np.zeros((0, 3))


def test_oracle_wall_distance(oracle_lib):
    """calc_wall_dists_parallel: sqrt of the minimum squared distance to any
    point of a bctype 2/20/21 region, plus small, at every point 1..n."""
    case = cases.small_plate_case()
    o = oracle_lib.Oracle(case)
    o.sa_setup()
    w = wall_points(case)
    assert len(w) > 0
    for nb, (x, y, z) in enumerate(case.xyz, start=1):
        p = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
        dx = p[:, None, 0] - w[None, :, 0]
        dy = p[:, None, 1] - w[None, :, 1]
        dz = p[:, None, 2] - w[None, :, 2]
        d2 = (dx * dx + dy * dy + dz * dz).min(axis=1)
        want = (np.sqrt(d2) + 1.0e-38).reshape(x.shape)
        got = interior(o.get("dist", nb), o.dims[nb - 1])
        np.testing.assert_array_equal(got, want)


def test_oracle_sa_init(oracle_lib):
    """init_SA: qke = muoo and vist = muoo*fv1(muoo) over -1..n+1."""
    case = cases.small_plate_case()
    o = oracle_lib.Oracle(case)
    o.sa_setup()
    kf3 = MUOO ** 3.0
    vt = MUOO * (kf3 / (kf3 + CV13))
    for nb in range(1, len(o.dims) + 1):
        ni, nj, nk = o.dims[nb - 1]
        q, v = o.get("qke", nb), o.get("vist", nb)
        sl = (slice(1, nk + 4), slice(1, nj + 4), slice(1, ni + 4))  # points -1..n+1
        assert np.all(q[sl] == MUOO)
        assert np.all(v[sl] == vt)


def sa_at_rest(r, qk, visl, vol, dtdt, dist, metr, reynolds, timedt_turb):
    """One model step for a fluid at rest with uniform qke, written out
    independently: the derivatives of qke and the velocity vanish, so the
    diffusion and convection terms and all LU-SGS off-diagonal products are
    zero; what remains is the source term, the diagonal (spec) and the
    update (turblence.f90:2567-2686, 218-259, 477-558, 585-623)."""
    cb1, cb2, cga, ki, cw2, cw3 = 0.1355, 0.622, 2.0 / 3.0, 0.419, 0.3, 2.0
    ki2, cw36, onesix = ki * ki, cw3 ** 6.0, 1.0 / 6.0
    cw1 = cb1 / ki / ki + (1.0 + cb2) / cga
    re = 1.0 / reynolds
    dn = np.where(dist > re, dist, re)
    dn2 = dn * dn
    reki2dn2 = (reynolds * ki2) * dn2
    kafan = (r * qk) / visl
    kf3 = np.power(kafan, 3.0)
    fv1 = kf3 / (kf3 + CV13)
    fv2 = 1.0 - kafan / (1.0 + kafan * fv1)
    sbar = 0.0 + (qk / reki2dn2) * fv2
    sbar = np.where(sbar > 1.0e-20, sbar, 1.0e-20)
    rbar = qk / (sbar * reki2dn2)
    rbar = np.where(rbar < 10.0, rbar, 10.0)
    gbar = rbar + (cw2 * rbar) * (np.power(rbar, 5.0) - 1.0)
    fw = gbar * np.power((1.0 + cw36) / (np.power(gbar, 6.0) + cw36), onesix)
    cpmu = cb1 * sbar
    cdmu = (cw1 * fw - 0.0) * qk / dn2 / reynolds
    dq = 0.0 - (r * ((cpmu * qk - cdmu * qk) + 0.0)) * vol
    sm = cpmu - 2.0 * cdmu
    spec = 0.0 - np.where(sm < 0.0, sm, 0.0) * vol
    spec = spec + 0.0 + 0.0 + 0.0 + 1.0 / (dtdt * timedt_turb)
    viseq = 1.5 * (visl / r + qk)
    ss = [metr[3 * d] * metr[3 * d] + metr[3 * d + 1] * metr[3 * d + 1] + metr[3 * d + 2] * metr[3 * d + 2]
          for d in range(3)]
    spec = spec + ((re * 2.0) * (viseq / vol)) * ((ss[0] + ss[1]) + ss[2])
    dq = (0.0 - dq) / spec
    qn = qk + dq / r
    return np.where(qn > 1.0e-21, qn, 1.0e-21)


def test_oracle_sa_at_rest(oracle_lib):
    case = cases.small_plate_case()
    o = oracle_lib.Oracle(case)
    for nb in range(1, len(o.dims) + 1):
        z = np.zeros_like(o.get("u", nb))
        for n in ("u", "v", "w"):
            o.set(n, nb, z)
    o.phase("initial_q_dq_c_t")
    o.phase("timestep")
    o.sa_setup(timedt_turb=2.0)
    o.phase("turbulence")
    names = ["kcx", "kcy", "kcz", "etx", "ety", "etz", "ctx", "cty", "ctz"]
    for nb in range(1, len(o.dims) + 1):
        ni, nj, nk = o.dims[nb - 1]
        c = (slice(4, nk + 2), slice(4, nj + 2), slice(4, ni + 2))  # interior points 2..n-1
        g = {n: o.get(n, nb)[c] for n in ["r", "visl", "vol", "dtdt", "dist"] + names}
        want = sa_at_rest(g["r"], MUOO, g["visl"], g["vol"], g["dtdt"], g["dist"], [g[n] for n in names],
                          case.params.reynolds, 2.0)
        np.testing.assert_allclose(o.get("qke", nb)[c], want, rtol=1e-14, atol=0)
        # vist follows qke at the interior points (cal_vist_SA)
        romu = g["r"] * o.get("qke", nb)[c]
        kf3 = np.power(romu / g["visl"], 3.0)
        np.testing.assert_allclose(o.get("vist", nb)[c], romu * (kf3 / (kf3 + CV13)), rtol=1e-14, atol=0)


def _region_geometry(r):
    """Face points of a BC record and its outward direction (s_lr3d)."""
    rng = [(abs(r[1 + 2 * d]), abs(r[2 + 2 * d])) for d in range(3)]
    lr = [0, 0, 0]
    for d in range(3):
        if rng[d][0] == rng[d][1]:
            lr[d] = -1 if rng[d][0] == 1 else 1
            break
    pts = [(i, j, k) for k in range(min(rng[2]), max(rng[2]) + 1) for j in range(min(rng[1]), max(rng[1]) + 1)
           for i in range(min(rng[0]), max(rng[0]) + 1)]
    return pts, lr


SA_BC_CASES = {
    "plate_small": lambda: cases.small_plate_case(),
    "plate_small_sym2d": lambda: cases.small_plate_case(nk=4),
    "supersonic_box": lambda: supersonic_box_case(),
    "channel_small": lambda: cases.small_channel_case(),
}


@pytest.mark.parametrize("name", list(SA_BC_CASES))
def test_oracle_sa_boundary_rules(oracle_lib, name):
    """The oracle's restatement of the model's one-layer qke/vist boundary
    rules (BC_*_turbulence and the interface copies), checked at every face
    point whose face, first ghost and interior neighbour no other region of
    the block touches: wall ghost = -interior and face = 0; symmetry ghost =
    interior and face = the mean; far field face and ghost = muoo where the
    boundary state flows in, else the interior value; inflow = muoo; outflow
    = interior; interface face = mean of the copied ghost and the interior."""
    case = SA_BC_CASES[name]()
    o = oracle_lib.Oracle(case)
    o.sa_setup()
    rng = np.random.default_rng(7)
    pre_q, pre_v = {}, {}
    for nb in range(1, len(o.dims) + 1):
        q = MUOO * (1.0 + rng.random(o.get("qke", nb).shape))
        v = 1e-6 * (1.0 + rng.random(q.shape))
        o.set("qke", nb, q); o.set("vist", nb, v)
        pre_q[nb], pre_v[nb] = q, v
    # switched off, boundary_all leaves qke alone: the rules are the only change
    o.sa_boundary_rules(False)
    o.phase("boundary_all")
    assert all(np.array_equal(o.get("qke", nb), pre_q[nb]) for nb in pre_q)
    for nb in pre_q:
        o.set("qke", nb, pre_q[nb]); o.set("vist", nb, pre_v[nb])
    o.sa_boundary_rules(True)
    o.phase("boundary_all")
    checked, ff_sides = {}, set()
    for nb in range(1, len(o.dims) + 1):
        regs = [r for r in case.regions if r[0] == nb]
        touched = {}
        geo = []
        for r in regs:
            pts, lr = _region_geometry(r)
            geo.append((r, pts, lr))
            for (i, j, k) in pts:
                for n in (0, 1):
                    p = (i + n * lr[0], j + n * lr[1], k + n * lr[2])
                    touched[p] = touched.get(p, 0) + 1
        q, v = o.get("qke", nb), o.get("vist", nb)
        U = [o.get(n, nb) for n in ("u", "v", "w")]
        A = lambda a, p: a[p[2] + 2, p[1] + 2, p[0] + 2]
        for r, pts, lr in geo:
            bt = int(r[7])
            sd = [d for d in range(3) if lr[d]][0]
            met = [o.get(n, nb) for n in (("kcx", "kcy", "kcz"), ("etx", "ety", "etz"), ("ctx", "cty", "ctz"))[sd]]
            for (i, j, k) in pts:
                f = (i, j, k)
                g = (i + lr[0], j + lr[1], k + lr[2])
                t = (i - lr[0], j - lr[1], k - lr[2])
                if touched.get(f) != 1 or touched.get(g) != 1 or t in touched:
                    continue
                qt = A(pre_q[nb], t)
                if bt == 2:
                    assert A(q, g) == -qt and A(q, f) == 0.0
                elif bt == 3:
                    assert A(q, g) == qt and A(q, f) == 0.5 * (qt + A(q, g))
                elif bt == 4:
                    ut = float(lr[sd]) * (A(met[0], f) * A(U[0], f) + A(met[1], f) * A(U[1], f) + A(met[2], f) * A(U[2], f))
                    want = MUOO if ut < 0.0 else qt
                    ff_sides.add(ut < 0.0)
                    assert A(q, f) == want and A(q, g) == want
                elif bt == 5:
                    assert A(q, f) == MUOO and A(q, g) == MUOO
                elif bt == 6:
                    assert A(q, f) == qt and A(q, g) == qt
                elif bt == -1:
                    assert A(q, f) == (A(q, g) + qt) * 0.5
                    assert A(v, f) == (A(v, g) + A(pre_v[nb], t)) * 0.5
                checked[bt] = checked.get(bt, 0) + 1
    types = set(int(x) for x in case.regions[:, 7])
    assert set(checked) == types, (checked, types)
    assert min(checked.values()) >= 4, checked
    if name == "plate_small":
        assert ff_sides == {True, False}  # both far-field branches seen


def test_oracle_sa_channel_steps(oracle_lib):
    """The 24-block SA channel (reduced size) runs through the oracle: SA set
    up with the case's settings, the model's boundary rules on, whole steps;
    the flow stays finite and the eddy viscosity grows from its free-stream
    value near the walls."""
    case = cases.small_channel_case()
    o = oracle_lib.Oracle(case)
    o.sa_setup(case.sa["timedt_turb"], case.sa["kmaxlim"])
    v0 = [interior(o.get("vist", nb), o.dims[nb - 1]).copy() for nb in range(1, len(o.dims) + 1)]
    hist = o.step(3)
    assert np.all(np.isfinite(hist))
    for nb in range(1, len(o.dims) + 1):
        d = o.dims[nb - 1]
        for n in ("r", "u", "p", "qke", "vist"):
            assert np.all(np.isfinite(interior(o.get(n, nb), d)))
    # lower-wall blocks: qke and vist vanish on the wall (BC_wall_turbulence),
    # and the eddy viscosity at the first off-wall points grows far above its
    # free-stream value
    lower = [nb for nb in range(1, case.nblocks + 1)
             if any((case.regions[:, 0] == nb) & (case.regions[:, 7] == 2) & (case.regions[:, 3] == 1) & (case.regions[:, 4] == 1))]
    assert len(lower) == 12
    for nb in lower:
        d = o.dims[nb - 1]
        q, v = interior(o.get("qke", nb), d), interior(o.get("vist", nb), d)
        assert np.all(q[:, 0, :] == 0.0) and np.all(v[:, 0, :] == 0.0)
        assert v[:, 1, :].mean() > 10.0 * v0[nb - 1][:, 1, :].mean()


# --------------------------------------------------------------------------
# GPU parity

def _pair(case):
    from oracle.pyoracle import Oracle
    from wcns_b200.solver import Wcns
    return Wcns(case), Oracle(case)


SA_CASES = {
    "plate_small": lambda: cases.small_plate_case(),
    "plate_small_sym2d": lambda: cases.small_plate_case(nk=4),
    "plate_small_roe42": lambda: cases.small_plate_case(nscheme=42),
    # no wall: the distance stays at its 1e30 start (sqrt 1e15)
    "vortex_viscous": lambda: with_params(cases.vortex_case(ni=33, nj=17, nk=9, nscheme=41, nflux=3), nvis=1),
}


@pytest.mark.gpu
@pytest.mark.parametrize("kmaxlim", [0.0, 3.0e-7])
@pytest.mark.parametrize("name", list(SA_CASES))
def test_sa_parity(name, kmaxlim):
    case = SA_CASES[name]()
    g, o = _pair(case)
    g.boundary_all(); o.phase("boundary_all")
    g.initial_q_dq_c_t(); o.phase("initial_q_dq_c_t")
    g.timestep_tgh(); o.phase("timestep")
    g.sa_setup(1.5, kmaxlim); o.sa_setup(1.5, kmaxlim)
    e = compare_fields(g, o, ["dist", "qke", "vist"], region="all")
    assert max(e.values()) == 0.0, e
    # a seeded non-uniform qke (ghosts included) so that every term is active
    rng = np.random.default_rng(11)
    for nb in range(1, len(o.dims) + 1):
        q = MUOO * (1.0 + 0.3 * rng.random(o.get("qke", nb).shape))
        g.set("qke", nb, q); o.set("qke", nb, q)
    q0 = o.get("qke", 1)
    for step in range(3):
        g.turbulence(); o.phase("turbulence")
        e = compare_fields(g, o, ["qke", "vist"], region="all")
        assert max(e.values()) <= TOL, (step, e)
    # the model moved qke
    d = o.dims[0]
    assert np.max(np.abs(interior(o.get("qke", 1), d) - interior(q0, d))) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["plate_small", "plate_small_sym2d"])
def test_sa_coupled(name):
    """With the model set up, the time step uses visl + vist (spectvist,
    LHS.f90:141-241), r_h_s_vis runs turbulence(nb) first (RHS.f90:22) and
    the viscous flux uses visl + vist and visl*cp/prl + vist*cp/prt; then
    whole steps through the step graph."""
    case = SA_CASES[name]()
    g, o = _pair(case)
    g.sa_setup(1.0, 0.0); o.sa_setup(1.0, 0.0)
    rng = np.random.default_rng(5)
    for nb in range(1, len(o.dims) + 1):
        q = MUOO * (1.0 + 50.0 * rng.random(o.get("qke", nb).shape))  # eddy viscosity of the order of visl
        g.set("qke", nb, q); o.set("qke", nb, q)
    g.boundary_all(); o.phase("boundary_all")
    g.initial_q_dq_c_t(); o.phase("initial_q_dq_c_t")
    g.timestep_tgh(); o.phase("timestep")
    e = compare_fields(g, o, ["dtdt", "srva", "srvb", "srvc"])
    assert max(e.values()) <= TOL, e
    g.r_h_s_vis(); o.phase("rhs_vis")
    e = compare_fields(g, o, ["qke", "vist"], region="all")
    e.update(compare_fields(g, o, ["dq1", "dq2", "dq3", "dq4", "dq5"]))
    assert max(e.values()) <= TOL, e
    hg = g.step(3)
    ho = o.step(3)
    np.testing.assert_allclose(hg, ho, rtol=1e-10, atol=0)
    e = compare_fields(g, o, ["r", "u", "v", "w", "p", "qke", "vist"])
    assert max(e.values()) <= 1e-10, e


@pytest.mark.gpu
def test_sa_errors():
    from wcns_b200.solver import Wcns, WcnsError
    g = Wcns(cases.small_plate_case())
    with pytest.raises(WcnsError) as ei:
        g.turbulence()
    assert ei.value.code == 1
    with pytest.raises(WcnsError) as ei:
        g.get("qke", 1)
    assert ei.value.code == 5
    with pytest.raises(WcnsError) as ei:
        g.sa_setup(0.0)
    assert ei.value.code == 1
    e = Wcns(cases.vortex_case(ni=17, nj=9, nk=9))  # inviscid: no visl
    with pytest.raises(WcnsError) as ei:
        e.sa_setup()
    assert ei.value.code == 5


# the model's qke/vist boundary rules on the device: cases that between them
# reach every rule (channel: cross-block interfaces, adiabatic walls, far
# field both ways, symmetry; viscous vortex: self-connected interfaces in
# place; viscous Mach-2 box: supersonic inflow and outflow)
SA_RULE_CASES = {
    "channel_small": lambda: cases.small_channel_case(),
    "plate_small": lambda: cases.small_plate_case(),
    "plate_small_sym2d": lambda: cases.small_plate_case(nk=4),
    "vortex_viscous": SA_CASES["vortex_viscous"],
    "supersonic_box_vis": lambda: with_params(supersonic_box_case(), nvis=1),
}

PHASES = [("boundary_all", "boundary_all"), ("initial_q_dq_c_t", "initial_q_dq_c_t"), ("timestep_tgh", "timestep"),
          ("r_h_s_vis", "rhs_vis"), ("communicate_dq_npp", "communicate_dq"), ("r_h_s_invis", "rhs_invis"),
          ("communicate_dq_npp", "communicate_dq"), ("l_h_s_tgh", "lhs"), ("communicate_pv_npp", "communicate_pv")]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(SA_RULE_CASES))
def test_sa_boundary_rules_parity(name):
    """boundary_all with the model set up: qke and vist at every point of
    the ghosted box (face points and first ghosts included) equal the
    oracle's after the rules, bitwise (copies, negations and means of equal
    inputs; the far-field branch is picked by the sign of a contravariant
    velocity, which agrees here); then a whole step phase by phase, each
    quantity within 1e-12 of its scale."""
    case = SA_RULE_CASES[name]()
    tt, km = (case.sa["timedt_turb"], case.sa["kmaxlim"]) if case.sa else (1.5, 0.0)
    g, o = _pair(case)
    g.sa_setup(tt, km); o.sa_setup(tt, km)
    rng = np.random.default_rng(17)
    for nb in range(1, len(o.dims) + 1):
        q = MUOO * (1.0 + 5.0 * rng.random(o.get("qke", nb).shape))
        v = 1e-5 * (1.0 + rng.random(q.shape))
        g.set("qke", nb, q); o.set("qke", nb, q)
        g.set("vist", nb, v); o.set("vist", nb, v)
    g.boundary_all(); o.phase("boundary_all")
    e = compare_fields(g, o, ["qke", "vist"], region="all")
    assert max(e.values()) == 0.0, e
    e = compare_fields(g, o, ["r", "u", "v", "w", "p"], region="all")
    assert max(e.values()) <= TOL, e
    for gp, op in PHASES[1:]:
        getattr(g, gp)(); o.phase(op)
        names = {"initial_q_dq_c_t": ["t"], "timestep_tgh": ["dtdt", "sra", "srva", "srvb", "srvc"],
                 "r_h_s_vis": ["qke", "vist", "dq1", "dq2", "dq3", "dq4", "dq5"],
                 "communicate_dq_npp": ["dq1", "dq2", "dq3", "dq4", "dq5"],
                 "r_h_s_invis": ["dq1", "dq2", "dq3", "dq4", "dq5"],
                 "l_h_s_tgh": ["r", "u", "v", "w", "p"], "communicate_pv_npp": ["r", "u", "v", "w", "p", "t"]}[gp]
        e = compare_fields(g, o, names, region="all" if gp == "r_h_s_vis" else "interior")
        assert max(e.values()) <= TOL, (gp, e)
    rg, ro = g.residual_curve(), o.residual()
    np.testing.assert_allclose(rg[0], ro[0], rtol=TOL, atol=0)
    np.testing.assert_allclose(rg[2], ro[2], rtol=TOL, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["channel_small", "vortex_viscous", "supersonic_box_vis"])
def test_sa_rules_graph_steps(name):
    """Whole steps through the step graph with the model and its boundary
    rules: residual history, conserved-variable fields and qke/vist."""
    case = SA_RULE_CASES[name]()
    tt, km = (case.sa["timedt_turb"], case.sa["kmaxlim"]) if case.sa else (1.5, 0.0)
    g, o = _pair(case)
    g.sa_setup(tt, km); o.sa_setup(tt, km)
    hg, ho = g.step(5), o.step(5)
    np.testing.assert_allclose(hg, ho, rtol=1e-12, atol=0)
    e = compare_fields(g, o, ["r", "u", "v", "w", "p", "qke", "vist"], region="all")
    assert max(e.values()) <= 1e-12, e


@pytest.mark.gpu
@pytest.mark.parametrize("narrow", [False, True])
def test_sa_wide_sweeps_graph_steps(narrow, monkeypatch):
    """The reduced channel with the wide cooperative sweeps (the path of the
    full channel), where the SA model's scalar LU-SGS runs on the same chunks:
    whole steps against the oracle, qke and vist included; with narrow
    chunks every j term crosses a ring between CTAs."""
    from oracle.pyoracle import Oracle
    from wcns_b200.solver import FLAG_SWEEP_WIDE, Wcns
    if narrow:
        monkeypatch.setenv("WCNS_WIDE_MIN_COLS", "1")
    case = cases.small_channel_case()
    g, o = Wcns(case, flags=FLAG_SWEEP_WIDE), Oracle(case)
    assert g.sweep_mode() == "wide"
    tt, km = case.sa["timedt_turb"], case.sa["kmaxlim"]
    g.sa_setup(tt, km); o.sa_setup(tt, km)
    hg, ho = g.step(5), o.step(5)
    np.testing.assert_allclose(hg, ho, rtol=1e-12, atol=0)
    e = compare_fields(g, o, ["r", "u", "v", "w", "p", "qke", "vist"], region="all")
    assert max(e.values()) <= 1e-12, e
