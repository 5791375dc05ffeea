"""Checks of the oracle that do not come from the oracle itself.

The reference cannot be built here and ships no test vectors, so the oracle
(a line-by-line C restatement of the Fortran) is pinned by properties of the
discretisation and by an independent restatement:

* order of accuracy: on a block periodic in all three directions (faces
  connected to themselves), with a smooth manufactured state, the inviscid
  residual dq/vol converges to the analytic flux divergence at the
  WCNS-E-5 interior order (about 5) away from the block ends and at the order
  of the 3rd-order end closures (about 3) over the whole block; the viscous
  residual converges to -(1/Re) div F_v (computed spectrally, exact for the
  trigonometric velocity field used) at the 4th order of its derivative
  operators in the interior.  A wrong coefficient or scaling in any stencil,
  flux or the viscous stress would stall the convergence at O(1);
* equivariance: exchanging the x and y axes of a block (grid, state and the
  u/v components) exchanges i and j and dq2/dq3 of every phase's result;
* the LU-SGS and symmetric Gauss-Seidel sweeps (l_h_s_tgh -> GS_PR_Single,
  LHS.f90:1-34, 381-577, 602-678, 756-828, 1559-1613, 1777-2046, getrkec_mml
  Sub1.f90:676-717) written out here again in plain Python, lexicographic
  point order, directly from the Fortran, and compared with the oracle's
  l_h_s on 9x7x5 blocks.
"""
import numpy as np
import pytest

from tests.helpers import interior, supersonic_box_case, with_params
from wcns_b200 import cases

GAMMA = 1.4


def periodic_box(n, nscheme=41, nflux=3, nvis=0, moo=0.5, reynolds=100.0):
    """One uniform Cartesian block on [0,1]^3 with n+1 points per direction,
    each face connected to the opposite face of the same block (period 1)."""
    dims = (n + 1,) * 3
    s = np.linspace(0.0, 1.0, n + 1)
    z, y, x = np.meshgrid(s, s, s, indexing="ij")
    rl = cases._RegionList()
    for a, b in (("i-", "i+"), ("j-", "j+"), ("k-", "k+")):
        rl.connect(1, cases._face(dims, a), 1, cases._face(dims, b))
    prm = cases.Params(moo=moo, nvis=nvis, nscheme=nscheme, nflux=nflux, reynolds=reynolds)
    return cases.Case("periodic_box", prm, [dims], [(x, y, z)], rl.array(), [cases.freestream_prim(prm, dims)], 1,
                      "periodic box")


def residual(oracle_lib, case, vis):
    o = oracle_lib.Oracle(case)
    o.phase("boundary_all")
    o.phase("initial_q_dq_c_t")
    o.phase("timestep")
    o.phase("rhs_vis" if vis else "rhs_invis")
    d = case.dims[0]
    vol = interior(o.get("vol", 1), d)
    out = [interior(o.get(f"dq{m}", 1), d) / vol for m in range(1, 6)]
    o.close()
    return out


def orders(errs):
    return [float(np.log2(errs[q] / errs[q + 1])) for q in range(len(errs) - 1)]


@pytest.mark.parametrize("nscheme,nflux", [(41, 3), (4, 1), (42, 2)])
def test_inviscid_residual_order(oracle_lib, nscheme, nflux):
    """Entropy wave: uniform velocity U and pressure, smooth density.  The
    Euler flux divergence is then U.grad(rho) * (1, U, |U|^2/2)."""
    k = 2.0 * np.pi
    U = (0.5, 0.3, 0.2)
    e_all, e_in = [], []
    for n in (12, 24, 48):
        case = periodic_box(n, nscheme=nscheme, nflux=nflux)
        x, y, z = case.xyz[0]
        r, u, v, w, p, t = case.prim[0]
        interior(r, case.dims[0])[...] = 1.0 + 0.1 * np.sin(k * x) * np.cos(k * y) + 0.05 * np.sin(k * z + 0.3)
        for a, val in zip((u, v, w), U):
            a[...] = val
        ddx = 0.1 * k * np.cos(k * x) * np.cos(k * y)
        ddy = -0.1 * k * np.sin(k * x) * np.sin(k * y)
        ddz = 0.05 * k * np.cos(k * z + 0.3)
        adv = U[0] * ddx + U[1] * ddy + U[2] * ddz
        v2 = U[0] ** 2 + U[1] ** 2 + U[2] ** 2
        exact = [adv, U[0] * adv, U[1] * adv, U[2] * adv, 0.5 * v2 * adv]
        dq = residual(oracle_lib, case, vis=False)
        inner = (slice(3, -4),) * 3  # at least 3 points from either end of every line
        e_all.append(max(float(np.max(np.abs(dq[m] - exact[m]))) for m in range(5)))
        e_in.append(max(float(np.max(np.abs(dq[m] - exact[m])[inner])) for m in range(5)))
    o_in, o_all = orders(e_in), orders(e_all)
    # the finest pair is in the asymptotic range; the coarsest not quite
    assert o_in[-1] >= 4.5 and min(o_in) >= 4.0, (o_in, e_in)
    assert min(o_all) >= 2.7, (o_all, e_all)
    assert e_in[-1] < 1e-4, e_in


def _spectral_d(f, axis):
    n = f.shape[axis]
    kk = 2.0 * np.pi * np.fft.fftfreq(n, d=1.0 / n)
    sh = [1, 1, 1]
    sh[axis] = n
    return np.real(np.fft.ifft(1j * kk.reshape(sh) * np.fft.fft(f, axis=axis), axis=axis))


def test_viscous_residual_order(oracle_lib):
    """Constant density and pressure (so T = 1, visl = 1 by Sutherland's law
    and no heat flux) and a trigonometric velocity field: dq/vol after
    r_h_s_vis must approach -(1/Re) div F_v, F_v = (0, tau, u.tau) with
    tau = grad u + grad u^T - 2/3 div u I."""
    k = 2.0 * np.pi
    e_all, e_in = [], []
    for n in (12, 24, 48):
        case = periodic_box(n, nvis=1)
        x, y, z = case.xyz[0]
        d = case.dims[0]
        r, u, v, w, p, t = case.prim[0]
        vel = [0.1 * np.sin(k * y) * np.cos(k * z), 0.08 * np.sin(k * z) * np.cos(k * x),
               0.05 * np.sin(k * x) * np.cos(k * y)]
        for a, val in zip((u, v, w), vel):
            interior(a, d)[...] = val
        dq = residual(oracle_lib, case, vis=True)
        # the exact operator on the n distinct points of the period
        V = [a[:-1, :-1, :-1] for a in vel]
        ax = (2, 1, 0)  # x, y, z are array axes 2, 1, 0
        g = [[_spectral_d(V[i], ax[j]) for j in range(3)] for i in range(3)]
        div = g[0][0] + g[1][1] + g[2][2]
        tau = [[g[i][j] + g[j][i] - (2.0 / 3.0) * div * (i == j) for j in range(3)] for i in range(3)]
        re = case.params.reynolds
        exact = [np.zeros_like(div)]
        exact += [-(1.0 / re) * sum(_spectral_d(tau[i][j], ax[j]) for j in range(3)) for i in range(3)]
        work = [sum(V[i] * tau[i][j] for i in range(3)) for j in range(3)]
        exact.append(-(1.0 / re) * sum(_spectral_d(work[j], ax[j]) for j in range(3)))
        got = [a[:-1, :-1, :-1] for a in dq]
        inner = (slice(3, -3),) * 3
        e_all.append(max(float(np.max(np.abs(got[m] - exact[m]))) for m in range(5)))
        e_in.append(max(float(np.max(np.abs(got[m] - exact[m])[inner])) for m in range(5)))
    o_in, o_all = orders(e_in), orders(e_all)
    assert min(o_in) >= 3.7, (o_in, e_in)
    assert min(o_all) >= 2.7, (o_all, e_all)


def _swap_xy_case(case):
    """The same block with the x and y axes exchanged: coordinates (y, x, z)
    and the i and j index directions swapped, u and v exchanged, BC records
    with their i and j ranges exchanged."""
    (ni, nj, nk), = case.dims
    x, y, z = case.xyz[0]
    sw = lambda a: np.ascontiguousarray(np.swapaxes(a, 1, 2))
    xyz = (sw(y), sw(x), sw(z))
    r, u, v, w, p, t = case.prim[0]
    prim = (sw(r), sw(v), sw(u), sw(w), sw(p), sw(t))
    regs = case.regions.copy()
    for base in (1, 8):
        regs[:, [base, base + 1, base + 2, base + 3]] = case.regions[:, [base + 2, base + 3, base, base + 1]]
    return cases.Case(case.name + "_swapped", case.params, [(nj, ni, nk)], [xyz], regs, [prim], case.nsteps, "")


@pytest.mark.parametrize("nvis", [0, 1])
def test_axis_exchange_equivariance(oracle_lib, nvis):
    """A smooth state varying in all five variables on the periodic box;
    every phase of a step on the x-y exchanged box gives the exchanged
    result (to round-off: the directions are summed in another order)."""
    case = periodic_box(12, nscheme=41, nflux=3, nvis=nvis)
    x, y, z = case.xyz[0]
    d = case.dims[0]
    k = 2.0 * np.pi
    r, u, v, w, p, t = case.prim[0]
    interior(r, d)[...] = 1.0 + 0.1 * np.sin(k * x) * np.cos(k * y) + 0.05 * np.sin(k * z)
    interior(u, d)[...] = 0.5 + 0.1 * np.cos(k * y) * np.sin(k * z)
    interior(v, d)[...] = 0.2 + 0.07 * np.sin(k * x + 0.4)
    interior(w, d)[...] = 0.1 * np.cos(k * x) * np.sin(k * y)
    interior(p, d)[...] = interior(p, d) * (1.0 + 0.05 * np.cos(k * z) * np.sin(k * x))
    swp = _swap_xy_case(case)
    o1, o2 = oracle_lib.Oracle(case), oracle_lib.Oracle(swp)
    sw = lambda a: np.swapaxes(a, 1, 2)
    names = {"dq2": "dq3", "dq3": "dq2", "u": "v", "v": "u"}
    phases = ["boundary_all", "initial_q_dq_c_t", "timestep"] + (["rhs_vis"] if nvis else []) + \
             ["rhs_invis", "communicate_dq", "lhs", "communicate_pv"]
    for ph in phases:
        o1.phase(ph)
        o2.phase(ph)
        dscale = max(float(np.max(np.abs(interior(o1.get(g, 1), d)))) for g in ("dq1", "dq2", "dq3", "dq4", "dq5"))
        for f in ("dq1", "dq2", "dq3", "dq4", "dq5", "r", "u", "v", "w", "p"):
            a = interior(o1.get(f, 1), d)
            b = sw(interior(o2.get(names.get(f, f), 1), d))
            scale = dscale if f.startswith("dq") else max(float(np.max(np.abs(a))), 0.5)
            assert float(np.max(np.abs(a - b))) <= 1e-12 * scale, (ph, f, float(np.max(np.abs(a - b))) / scale)


# ---------------------------------------------------------------------------
# LU-SGS + symmetric Gauss-Seidel, restated from LHS.f90 in plain Python

def _mxdq_std(prim, gykb, dq, rad, npn, moo):
    """mxdq_std, LHS.f90:756-828 (nl = 5, perfect gas: gettmhmgm_ns,
    GasModel.f90:411-426)."""
    rm, um, vm, wm, pm = prim
    gama = GAMMA
    hint = gama / (gama - 1.0) * pm / rm
    c2 = gama * pm / rm
    cm = np.sqrt(c2)
    v2 = um * um + vm * vm + wm * wm
    hm = hint + 0.5 * v2
    nx, ny, nz, nt = gykb
    ct = nx * um + ny * vm + nz * wm + nt
    cgm = max(np.sqrt(nx * nx + ny * ny + nz * nz), 1.0e-30)
    l1 = ct
    l4 = ct + cm * cgm
    l5 = ct - cm * cgm
    l1 = 0.5 * (l1 + npn * rad)
    l4 = 0.5 * (l4 + npn * rad)
    l5 = 0.5 * (l5 + npn * rad)
    x1 = (2.0 * l1 - l4 - l5) / (2.0 * c2)
    x2 = (l4 - l5) / (2.0 * cm)
    cgm1 = 1.0 / cgm
    nx, ny, nz = nx * cgm1, ny * cgm1, nz * cgm1
    ct = (ct - nt) * cgm1
    ae = gama - 1.0
    af = 0.5 * ae * v2
    dc = ct * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3]
    dh = af * dq[0] - ae * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4])
    c2dc = c2 * dc
    return np.array([l1 * dq[0] - dh * x1 - dc * x2,
                     l1 * dq[1] + (nx * c2dc - um * dh) * x1 + (nx * dh - um * dc) * x2,
                     l1 * dq[2] + (ny * c2dc - vm * dh) * x1 + (ny * dh - vm * dc) * x2,
                     l1 * dq[3] + (nz * c2dc - wm * dh) * x1 + (nz * dh - wm * dc) * x2,
                     l1 * dq[4] + (ct * c2dc - hm * dh) * x1 + (ct * dh - hm * dc) * x2])


class _Block:
    """Fields of one block indexed by the reference's (i, j, k)."""

    def __init__(self, o, nb, case):
        self.ni, self.nj, self.nk = case.dims[nb - 1]
        g = lambda n: o.get(n, nb)
        self.prim = [g(n) for n in ("r", "u", "v", "w", "p")]
        self.met = [[g(n) for n in grp] for grp in (("kcx", "kcy", "kcz"), ("etx", "ety", "etz"), ("ctx", "cty", "ctz"))]
        self.sr = [g("sra"), g("srb"), g("src")]
        self.srv = [g("srva"), g("srvb"), g("srvc")]
        self.dtdt = g("dtdt")
        self.dq = np.stack([g(f"dq{m}") for m in range(1, 6)])  # ghosted, (5, nk+6, nj+6, ni+6)

    def at(self, a, i, j, k):
        return a[k + 2, j + 2, i + 2]

    def getprim(self, i, j, k):
        return [self.at(a, i, j, k) for a in self.prim]

    def getrkec(self, i, j, k, d):
        """getrkec_mml, Sub1.f90:676-717: metrics of direction d at (i,j,k)
        with the index clamped into the block; nt = 0 (steady grid)."""
        i1 = min(max(i, 1), self.ni)
        j1 = min(max(j, 1), self.nj)
        k1 = min(max(k, 1), self.nk)
        return [self.at(a, i1, j1, k1) for a in self.met[d]] + [0.0]

    def rad(self, i, j, k, dijk):
        """getrarbrc, LHS.f90:647-678, method 1."""
        c = [min(max(v + dijk, 1), n) for v, n in zip((i, j, k), (self.ni, self.nj, self.nk))]
        return (self.at(self.sr[0], c[0], j, k), self.at(self.sr[1], i, c[1], k), self.at(self.sr[2], i, j, c[2]))

    def coed(self, i, j, k, nvis):
        """getcoed, LHS.f90:602-645 (beta = wmig = 1, no dual time step)."""
        rad_ns = self.at(self.sr[0], i, j, k) + self.at(self.sr[1], i, j, k) + self.at(self.sr[2], i, j, k)
        if nvis:
            rad_ns = rad_ns + self.at(self.srv[0], i, j, k) + self.at(self.srv[1], i, j, k) + self.at(self.srv[2], i, j, k)
        ct = 1.0 / self.at(self.dtdt, i, j, k)
        return 1.0 / (ct + 1.0 * 1.0 * rad_ns)

    def dqv(self, i, j, k):
        return self.dq[:, k + 2, j + 2, i + 2]


def _neigh(i, j, k, d, s):
    c = [i, j, k]
    c[d] += s
    return tuple(c)


def lu_sgs_python(b, nvis, moo):
    """GS_PR_Single (LHS.f90:1559-1613): lusgs_l, lusgs_u, gs_pr_l, gs_pr_u
    over the interior points 1..n, in the Fortran loop order."""
    rhs_nb = b.dq.copy()
    fwd = [(i, j, k) for k in range(1, b.nk + 1) for j in range(1, b.nj + 1) for i in range(1, b.ni + 1)]
    bwd = fwd[::-1]
    n = (b.ni, b.nj, b.nk)
    # lusgs_l (LHS.f90:381-478): lower neighbours, dq(i-1) as it stands
    for (i, j, k) in fwd:
        ra = b.rad(i, j, k, -1)
        parts = [_mxdq_std(b.getprim(*_neigh(i, j, k, d, -1)), b.getrkec(*_neigh(i, j, k, d, -1), d),
                           b.dqv(*_neigh(i, j, k, d, -1)), ra[d], 1, moo) for d in range(3)]
        rhs0 = 1.0 * (parts[0] + parts[1] + parts[2])
        if nvis:
            rv = [b.at(b.srv[d], *_neigh(i, j, k, d, -1)) for d in range(3)]
            rhs0 = rhs0 + 0.5 * (rv[0] * b.dqv(*_neigh(i, j, k, 0, -1)) + rv[1] * b.dqv(*_neigh(i, j, k, 1, -1))
                                 + rv[2] * b.dqv(*_neigh(i, j, k, 2, -1)))
        b.dq[:, k + 2, j + 2, i + 2] = (-b.dqv(i, j, k) + rhs0) * b.coed(i, j, k, nvis)
    # lusgs_u (480-577): upper neighbours
    for (i, j, k) in bwd:
        ra = b.rad(i, j, k, 1)
        parts = [_mxdq_std(b.getprim(*_neigh(i, j, k, d, 1)), b.getrkec(*_neigh(i, j, k, d, 1), d),
                           b.dqv(*_neigh(i, j, k, d, 1)), ra[d], -1, moo) for d in range(3)]
        rhs0 = 1.0 * (parts[0] + parts[1] + parts[2])
        if nvis:
            rv = [b.at(b.srv[d], *_neigh(i, j, k, d, 1)) for d in range(3)]
            rhs0 = rhs0 - 0.5 * (rv[0] * b.dqv(*_neigh(i, j, k, 0, 1)) + rv[1] * b.dqv(*_neigh(i, j, k, 1, 1))
                                 + rv[2] * b.dqv(*_neigh(i, j, k, 2, 1)))
        b.dq[:, k + 2, j + 2, i + 2] = b.dqv(i, j, k) - rhs0 * b.coed(i, j, k, nvis)
    # gs_pr_l (1777-1866) and gs_pr_u (1956-2046): both sides, zero dq
    # outside the block, no viscous off-diagonal terms
    for order in (fwd, bwd):
        for (i, j, k) in order:
            c = (i, j, k)
            lo, hi = [], []
            for d in range(3):
                pl, ph = _neigh(i, j, k, d, -1), _neigh(i, j, k, d, 1)
                dl = np.zeros(5) if c[d] == 1 else b.dqv(*pl)
                dh = np.zeros(5) if c[d] == n[d] else b.dqv(*ph)
                lo.append((pl, dl))
                hi.append((ph, dh))
            ra_l, ra_u = b.rad(i, j, k, -1), b.rad(i, j, k, 1)
            dl = [_mxdq_std(b.getprim(*lo[d][0]), b.getrkec(*lo[d][0], d), lo[d][1], ra_l[d], 1, moo) for d in range(3)]
            du = [_mxdq_std(b.getprim(*hi[d][0]), b.getrkec(*hi[d][0], d), hi[d][1], ra_u[d], -1, moo) for d in range(3)]
            rhs0 = 1.0 * (dl[0] + dl[1] + dl[2] - du[0] - du[1] - du[2])
            b.dq[:, k + 2, j + 2, i + 2] = (rhs0 - rhs_nb[:, k + 2, j + 2, i + 2]) * b.coed(i, j, k, nvis)
    return b.dq


def _zero_physical_faces(dq, case, nb):
    """set_nonconnect_boundary_dq_0 (CIC.f90:2-17, 482-506): dq = 0 at the
    points of the block's physical-boundary regions."""
    for r in case.regions:
        if r[0] != nb or r[7] <= 0:
            continue
        lo = [min(abs(r[1 + 2 * m]), abs(r[2 + 2 * m])) for m in range(3)]
        hi = [max(abs(r[1 + 2 * m]), abs(r[2 + 2 * m])) for m in range(3)]
        dq[:, lo[2] + 2:hi[2] + 3, lo[1] + 2:hi[1] + 3, lo[0] + 2:hi[0] + 3] = 0.0


LHS_CASES = {
    "vortex_9x7x5_viscous": lambda: with_params(cases.vortex_case(ni=9, nj=7, nk=5, nscheme=41, nflux=3), nvis=1),
    "vortex_9x7x5_euler": lambda: cases.vortex_case(ni=9, nj=7, nk=5, nscheme=4, nflux=1),
    "supersonic_box_9x7x5": lambda: supersonic_box_case(ni=9, nj=7, nk=5),
    "plate_block_viscous": lambda: _single_plate_block(),
}


def _single_plate_block():
    """A 9x7x5 viscous block with an isothermal wall at j = 1, far field at
    j = nj and i = ni, symmetry at the k faces and supersonic-like inflow
    replaced by far field at i = 1, and a seeded non-uniform state."""
    dims = (9, 7, 5)
    s = np.linspace(0.0, 1.0, 9)
    t = np.linspace(0.0, 1.0, 7) ** 2 * 0.5
    q = np.linspace(0.0, 0.2, 5)
    z, y, x = np.meshgrid(q, t, s, indexing="ij")
    rl = cases._RegionList()
    rl.add(1, cases._face(dims, "j-"), 2)
    for f in ("j+", "i-", "i+"):
        rl.add(1, cases._face(dims, f), 4)
    rl.add(1, cases._face(dims, "k-"), 3)
    rl.add(1, cases._face(dims, "k+"), 3)
    prm = cases.Params(moo=0.4, nvis=1, nscheme=41, nflux=3, reynolds=1.0e3, twall=300.0)
    prim = cases.freestream_prim(prm, dims)
    rng = np.random.default_rng(9)
    for f in (0, 1, 2, 4):
        interior(prim[f], dims)[...] *= 1.0 + 0.05 * rng.random((5, 7, 9))
    return cases.Case("plate_block", prm, [dims], [(x, y, z)], rl.array(), [tuple(prim)], 1, "")


@pytest.mark.parametrize("name", list(LHS_CASES))
def test_lusgs_sweeps_against_python_restatement(oracle_lib, name):
    case = LHS_CASES[name]()
    o = oracle_lib.Oracle(case)
    for ph in ("boundary_all", "initial_q_dq_c_t", "timestep") + (("rhs_vis",) if case.params.nvis else ()) + \
              ("rhs_invis", "communicate_dq"):
        o.phase(ph)
    b = _Block(o, 1, case)
    _zero_physical_faces(b.dq, case, 1)
    want = lu_sgs_python(b, case.params.nvis, case.params.moo)
    _zero_physical_faces(want, case, 1)
    o.phase("lhs")
    d = case.dims[0]
    got = np.stack([interior(o.get(f"dq{m}", 1), d) for m in range(1, 6)])
    ref = np.stack([interior(want[m], d) for m in range(5)])
    scale = float(np.max(np.abs(ref)))
    assert scale > 0.0
    err = float(np.max(np.abs(got - ref))) / scale
    assert err <= 1e-13, err
