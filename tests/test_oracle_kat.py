"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests or golden vectors, so the oracle is pinned by
properties its operators must have by construction:
  * VALUE_HALF_NODE is exact for cubics in the interior and for quadratics
    at the ends (WCNSE5.f90:799-852);
  * FLUX_DXYZ is exact for the derivative of a degree-6 polynomial flux in
    the interior (WCNSE5.f90:209-254);
  * the Roe flux of two equal states is the physical flux, and the
    Steger-Warming split fluxes sum to it when efix = 0 (flux.f90:2-244);
  * the WCNS line scheme of a uniform state gives zero residual;
  * a uniform free stream on a curved grid with far-field faces stays a
    solution: the GCL metrics (WCNSE5.f90:1478-1728) make the residual vanish
    to round-off, inviscid and viscous (for nscheme 41 away from the faces).
"""
import ctypes as C

import numpy as np
import pytest

from wcns_b200 import cases

GAMMA = 1.4


@pytest.fixture(scope="module")
def L(oracle_lib):
    lib = oracle_lib.lib()
    dp = C.POINTER(C.c_double)
    lib.orc_value_half_node.argtypes = [C.c_int, C.c_int, dp, dp]
    lib.orc_flux_dxyz.argtypes = [C.c_int, C.c_int, dp, dp]
    lib.orc_fluxes.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, dp]
    lib.orc_wcns_line.argtypes = [C.c_void_p, C.c_int, dp, dp, dp]
    lib.orc_wcns_line.restype = C.c_int
    return lib


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def test_value_half_node_polynomial_exactness(L):
    ni = 12
    x = np.arange(1, ni + 1, dtype=np.float64)
    xh = np.arange(0, ni + 1, dtype=np.float64) + 0.5
    cubic = lambda s: 0.3 - 1.1 * s + 0.07 * s ** 2 - 0.002 * s ** 3
    quad = lambda s: 0.3 - 1.1 * s + 0.07 * s ** 2
    for fun, rng in ((cubic, slice(2, ni - 1)), (quad, slice(0, ni + 1))):
        q = np.ascontiguousarray(fun(x))
        qh = np.zeros(ni + 1)
        L.orc_value_half_node(1, ni, _p(q), _p(qh))
        np.testing.assert_allclose(qh[rng], fun(xh)[rng], rtol=1e-13, atol=1e-13)


def test_flux_dxyz_sixth_order_interior(L):
    ni = 16
    xh = np.arange(0, ni + 1, dtype=np.float64) + 0.5  # half nodes i+1/2, i = 0..ni
    c = [0.2, -0.5, 0.03, 0.004, -1e-4, 2e-6, -1e-8]
    f = np.ascontiguousarray(sum(ck * xh ** k for k, ck in enumerate(c)))
    dfx = lambda s: sum(k * ck * s ** (k - 1) for k, ck in enumerate(c) if k)
    df = np.zeros(ni)
    L.orc_flux_dxyz(1, ni, _p(f), _p(df))
    nodes = np.arange(1, ni + 1, dtype=np.float64)
    np.testing.assert_allclose(df[2:ni - 2], dfx(nodes)[2:ni - 2], rtol=1e-11, atol=1e-11)


def _prm(oracle_lib, efix=0.1):
    p = cases.Params(moo=0.5, efix=efix)
    return oracle_lib.params_struct(p)


def test_roe_of_equal_states_is_physical_flux(L, oracle_lib):
    rng = np.random.default_rng(1)
    prm = _prm(oracle_lib)
    for _ in range(20):
        q = np.ascontiguousarray([rng.uniform(0.5, 2.0), *rng.uniform(-1, 1, 3), rng.uniform(1.0, 4.0)])
        n4 = np.ascontiguousarray([*rng.uniform(-1, 1, 3), 0.0])
        f_phys, f_roe = np.zeros(5), np.zeros(5)
        L.orc_fluxes(C.byref(prm), 0, _p(q), _p(q), _p(n4), _p(f_phys))
        L.orc_fluxes(C.byref(prm), 3, _p(q), _p(q), _p(n4), _p(f_roe))
        np.testing.assert_allclose(f_roe, f_phys, rtol=1e-13, atol=1e-13 * np.abs(f_phys).max())


def test_steger_warming_split_sums_to_flux(L, oracle_lib):
    rng = np.random.default_rng(2)
    prm = _prm(oracle_lib, efix=0.0)
    for _ in range(20):
        q = np.ascontiguousarray([rng.uniform(0.5, 2.0), *rng.uniform(-1, 1, 3), rng.uniform(1.0, 4.0)])
        n4 = np.ascontiguousarray([*rng.uniform(-1, 1, 3), 0.0])
        f_phys, f_sw = np.zeros(5), np.zeros(5)
        L.orc_fluxes(C.byref(prm), 0, _p(q), _p(q), _p(n4), _p(f_phys))
        L.orc_fluxes(C.byref(prm), 1, _p(q), _p(q), _p(n4), _p(f_sw))
        np.testing.assert_allclose(f_sw, f_phys, rtol=1e-12, atol=1e-12 * np.abs(f_phys).max())


def test_van_leer_split_sums_to_flux(L, oracle_lib):
    """flux_vanleer of equal states: the positive and negative parts of Van
    Leer's splitting add up to the physical flux, subsonic and supersonic."""
    rng = np.random.default_rng(4)
    prm = _prm(oracle_lib)
    seen = set()
    for _ in range(40):
        q = np.ascontiguousarray([rng.uniform(0.5, 2.0), *rng.uniform(-2.5, 2.5, 3), rng.uniform(0.5, 4.0)])
        n4 = np.ascontiguousarray([*rng.uniform(-1, 1, 3), 0.0])
        mach = abs(q[1:4] @ n4[:3]) / np.linalg.norm(n4[:3]) / np.sqrt(1.4 * q[4] / q[0])
        seen.add(mach >= 1.0)
        f_phys, f_vl = np.zeros(5), np.zeros(5)
        L.orc_fluxes(C.byref(prm), 0, _p(q), _p(q), _p(n4), _p(f_phys))
        L.orc_fluxes(C.byref(prm), 2, _p(q), _p(q), _p(n4), _p(f_vl))
        np.testing.assert_allclose(f_vl, f_phys, rtol=1e-12, atol=1e-12 * np.abs(f_phys).max())
    assert seen == {True, False}


@pytest.mark.parametrize("nscheme,nflux", [(4, 1), (41, 1), (42, 1), (4, 2), (41, 2), (42, 2), (4, 3), (41, 3), (42, 3)])
def test_wcns_line_uniform_state_has_zero_residual(L, oracle_lib, nscheme, nflux):
    ni = 11
    p = cases.Params(moo=0.5, nscheme=nscheme, nflux=nflux)
    prm = oracle_lib.params_struct(p)
    roo, uoo, voo, woo, poo = p.freestream()
    q = np.ascontiguousarray(np.repeat([roo, uoo, voo, woo, poo], ni + 6).reshape(5, ni + 6))
    nx = np.ascontiguousarray(np.tile([0.7, 0.2, -0.1, 0.0], ni + 1))
    df = np.zeros(5 * ni)
    assert L.orc_wcns_line(C.byref(prm), ni, _p(q), _p(nx), _p(df)) == 0
    assert np.abs(df).max() <= 1e-13


@pytest.mark.parametrize("nscheme", [41, 42])
@pytest.mark.parametrize("nflux", [1, 2, 3])
def test_wcns_line_sections_keep_a_uniform_state(L, oracle_lib, nscheme, nflux):
    """With both line ends flagged as physical boundaries (third ghost layer
    density negative, as the wall and far-field conditions leave it), the
    boundary sections of nscheme 41 and 42 run; their end states reproduce
    a constant, so a uniform state still has a zero residual."""
    ni = 13
    p = cases.Params(moo=0.5, nscheme=nscheme, nflux=nflux)
    prm = oracle_lib.params_struct(p)
    roo, uoo, voo, woo, poo = p.freestream()
    q = np.repeat([roo, uoo, voo, woo, poo], ni + 6).reshape(5, ni + 6)
    q[0, 0] = -roo
    q[0, ni + 5] = -roo
    q = np.ascontiguousarray(q)
    nx = np.ascontiguousarray(np.tile([0.7, 0.2, -0.1, 0.0], ni + 1))
    df = np.zeros(5 * ni)
    assert L.orc_wcns_line(C.byref(prm), ni, _p(q), _p(nx), _p(df)) == 0
    assert np.abs(df).max() <= 1e-12


def wavy_freestream_case(nvis, nscheme=41, nflux=3, dims=(17, 13, 9)):
    """One curved block, all six faces far field, uniform free stream."""
    ni, nj, nk = dims
    prm = cases.Params(moo=0.5, attack=5.0, nvis=nvis, nscheme=nscheme, nflux=nflux, reynolds=1e4)
    s = np.linspace(0.0, 1.0, ni)
    t = np.linspace(0.0, 1.0, nj)
    u = np.linspace(0.0, 1.0, nk)
    zz, yy, xx = np.meshgrid(u, t, s, indexing="ij")
    x = 2.0 * xx + 0.08 * np.sin(2 * np.pi * yy) * np.sin(np.pi * zz)
    y = 1.5 * yy + 0.06 * np.sin(2 * np.pi * xx) + 0.03 * zz * xx
    z = 1.0 * zz + 0.05 * np.sin(np.pi * xx) * np.cos(np.pi * yy)
    rl = cases._RegionList()
    for face in ("i-", "i+", "j-", "j+", "k-", "k+"):
        rl.add(1, cases._face(dims, face), 4)
    prim = cases.freestream_prim(prm, dims)
    return cases.Case("wavy", prm, [dims], [(x, y, z)], rl.array(), [tuple(prim)], 1, "free stream on a curved block")


@pytest.mark.parametrize("nvis", [0, 1])
@pytest.mark.parametrize("nscheme,nflux", [(4, 1), (41, 3)])
def test_freestream_preservation_curved_grid(oracle_lib, nvis, nscheme, nflux):
    """nscheme 4 keeps the free stream on every point; the boundary closures
    of nscheme 41 (WCNSE5.f90:2087-2759) are not metric-consistent, so there
    the bar holds three points away from the faces."""
    case = wavy_freestream_case(nvis, nscheme, nflux)
    o = oracle_lib.Oracle(case)
    for ph in ("boundary_all", "initial_q_dq_c_t", "timestep"):
        o.phase(ph)
    if nvis:
        o.phase("rhs_vis")
    o.phase("rhs_invis")
    dims = case.dims[0]
    # flux scale: rho * |U| * |grad xi| * vol ~ one cell face area
    area = np.abs(cases.interior(o.get("kcx", 1), dims)).max()
    for m in range(1, 6):
        dq = cases.interior(o.get(f"dq{m}", 1), dims)
        if nscheme == 41:
            dq = dq[3:-3, 3:-3, 3:-3]
        assert np.abs(dq).max() <= 1e-11 * area, (m, np.abs(dq).max())


def test_force_of_uniform_pressure_on_flat_wall(oracle_lib):
    """force_dif on the small plate with a uniform excess pressure dp and no
    viscosity: the wall (y = 0, normal +y, s_lr = -1) carries 2*dp*area in
    -y, centred at the wall's centroid (PostProcess.f90:1505-1824)."""
    case = cases.small_plate_case()
    case.params.nvis = 0
    o = oracle_lib.Oracle(case)
    poo = case.params.freestream()[4]
    dp = 0.1
    for nb in range(1, len(case.dims) + 1):
        o.set("p", nb, np.full_like(o.get("p", nb), poo + dp))
    area, mx, mz = 0.0, 0.0, 0.0
    for r in case.regions:
        if r[7] != 2:
            continue
        x, y, z = case.xyz[r[0] - 1]
        sl = tuple(slice(r[2 * d + 1] - 1, r[2 * d + 2]) for d in (2, 1, 0))
        assert np.abs(y[sl]).max() == 0.0
        a = (x[sl].max() - x[sl].min()) * (z[sl].max() - z[sl].min())
        area += a
        mx += a * 0.5 * (z[sl].max() + z[sl].min())
        mz += a * 0.5 * (x[sl].max() + x[sl].min())
    f = o.force(sref=1.0, lfref=1.0)
    assert f["cfy"] == pytest.approx(-2 * dp * area, rel=1e-13)
    assert abs(f["cfx"]) < 1e-15 and abs(f["cfz"]) < 1e-15
    assert f["cmx"] == pytest.approx(2 * dp * mx, rel=1e-12)
    assert f["cmz"] == pytest.approx(-2 * dp * mz, rel=1e-12)


def test_flux_dxyz_interior_telescopes(L):
    """Discrete conservation of the interior difference: over the points
    3..n-2 the 6th-order FLUX_DXYZ is the difference of a numerical flux,
    G(l) = 2250 f(l) - 125 (f(l-1)+f(l)+f(l+1)) + 9 (f(l-2)+...+f(l+2)), so any
    sum of consecutive interior differences telescopes to (G(b) - G(a-1))/1920
    for random half-node values.  (The one-sided closures at l = 1, 2, n-1, n,
    which the reference applies at every block end, interfaces included, do
    not telescope: a periodic box's summed residual is not zero.)"""
    rng = np.random.default_rng(7)
    ni = 24
    f = np.ascontiguousarray(rng.standard_normal(ni + 1))
    df = np.zeros(ni)
    L.orc_flux_dxyz(1, ni, _p(f), _p(df))
    G = lambda l: 2250 * f[l] - 125 * (f[l - 1] + f[l] + f[l + 1]) + 9 * (f[l - 2] + f[l - 1] + f[l] + f[l + 1] + f[l + 2])
    for a, b in ((3, ni - 2), (5, 11), (4, 4)):
        lhs = float(np.sum(df[a - 1:b]))
        rhs = (G(b) - G(a - 1)) / 1920.0
        assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(rhs)), (a, b, lhs, rhs)
