"""Tangent and adjoint of the inviscid residual, and the LU-SGS operator pair
(k_adjoint.cu through wcns_rhs_invis_tangent / wcns_rhs_invis_adjoint /
wcns_lusgs_operator / wcns_adjoint_iterate).

r is the inviscid residual (dq of r_h_s_invis) as a function of the ghosted
prim state; the checks:
  * dot products <lam, (dr/dq) v> = <(dr/dq)^T lam, v> to round-off, with v
    over every point, ghosts included (the unfolded adjoint);
  * the tangent against central differences of the FP64 residual kernel
    with the ghosts held (second-order truncation, step 1e-6);
  * on a box periodic in every direction (its ghosts are all interface
    copies), the folded adjoint against central differences of the
    residual with the ghosts refilled by the boundary phase;
  * <y, P b> = <P^T y, b> for the LU-SGS operator, and P b against a NumPy
    restatement of lusgs_l / lusgs_u (LHS.f90:381-577, mxdq_std 756-828);
  * each step of the adjoint fixed point psi <- psi + Z P^T Z (r_Q^T psi + g)
    is that formula, assembled here from the separate operators."""
import numpy as np
import pytest

from tests.helpers import interior, perturbed, supersonic_box_case, with_params
from wcns_b200 import cases

pytestmark = pytest.mark.gpu


def periodic_box(n=12, nflux=3, amp=0.05):
    """A uniform block on [0,1]^3 with every face connected to the opposite
    one (period 1), carrying a smooth periodic density / pressure / velocity
    perturbation of the Mach-0.5 free stream."""
    dims = (n + 1,) * 3
    s = np.linspace(0.0, 1.0, n + 1)
    z, y, x = np.meshgrid(s, s, s, indexing="ij")
    rl = cases._RegionList()
    for a, b in (("i-", "i+"), ("j-", "j+"), ("k-", "k+")):
        rl.connect(1, cases._face(dims, a), 1, cases._face(dims, b))
    prm = cases.Params(moo=0.5, nvis=0, nscheme=4, nflux=nflux)
    prim = [a.copy() for a in cases.freestream_prim(prm, dims)]
    w = 2.0 * np.pi
    sl = (slice(3, 3 + n + 1),) * 3
    bump = np.sin(w * x) * np.cos(w * y) * np.sin(w * z + 0.3)
    prim[0][sl] *= 1.0 + amp * bump
    prim[4][sl] *= 1.0 + 0.5 * amp * np.cos(w * x + 0.1) * np.sin(w * y)
    prim[1][sl] += amp * np.sin(w * z)
    prim[2][sl] += amp * np.cos(w * x)
    return cases.Case("periodic_box", prm, [dims], [(x, y, z)], rl.array(), [tuple(prim)], 1, "periodic box")


def make(name):
    if name == "vortex_sw":
        return cases.vortex_case(ni=25, nj=13, nk=9, nscheme=4, nflux=1, nsteps=1)
    if name == "vortex_roe":
        return cases.vortex_case(ni=25, nj=13, nk=9, nscheme=4, nflux=3, nsteps=1)
    if name == "plate_euler":
        return perturbed(with_params(cases.small_plate_case(), nvis=0, nscheme=4))
    if name == "box_roe":
        return supersonic_box_case(nscheme=4, nflux=3)
    if name == "periodic":
        return periodic_box()
    raise KeyError(name)


CASES = ["vortex_sw", "vortex_roe", "plate_euler", "box_roe", "periodic"]


def ctx(case, phases=False):
    from wcns_b200.solver import Wcns
    g = Wcns(case)
    g.boundary_all()
    if phases:
        g.initial_q_dq_c_t()
        g.timestep_tgh()
    return g


def rand_fields(case, rng, ghosts, scale=None):
    out = []
    for nb, (ni, nj, nk) in enumerate(case.dims, start=1):
        f = []
        for m in range(5):
            a = rng.standard_normal((nk + 6, nj + 6, ni + 6))
            if scale is not None:
                a *= scale[m]
            if not ghosts:
                b = np.zeros_like(a)
                b[3:3 + nk, 3:3 + nj, 3:3 + ni] = a[3:3 + nk, 3:3 + nj, 3:3 + ni]
                a = b
            f.append(a)
        out.append(f)
    return out


def dot(case, a, b, ghosts):
    s = 0.0
    for nb, d in enumerate(case.dims):
        for m in range(5):
            x, y = a[nb][m], b[nb][m]
            if not ghosts:
                x, y = interior(x, d), interior(y, d)
            s += float(np.sum(x * y))
    return s


def norm(case, a, ghosts):
    return dot(case, a, a, ghosts) ** 0.5


def residual(g, case, prims, refill):
    """dq of the FP64 residual kernel at the given ghosted prim arrays."""
    for nb, p in enumerate(prims, start=1):
        g.set_prim(nb, p)
    if refill:
        g.boundary_all()
    g.initial_q_dq_c_t()
    g.r_h_s_invis()
    return [[g.get(f"dq{m}", nb) for m in range(1, 6)] for nb in range(1, case.nblocks + 1)]


def state_scales(g, case):
    return [max(float(np.max(np.abs(interior(g.get(f, nb), case.dims[nb - 1])))) for nb in range(1, case.nblocks + 1))
            for f in ("r", "u", "v", "w", "p")]


@pytest.mark.parametrize("name", CASES)
def test_tangent_adjoint_dot_product(name):
    case = make(name)
    g = ctx(case)
    rng = np.random.default_rng(11)
    sc = state_scales(g, case)
    sc = [max(s, 0.1) for s in sc]
    v = rand_fields(case, rng, ghosts=True, scale=sc)
    lam = rand_fields(case, rng, ghosts=False)
    for nb in range(1, case.nblocks + 1):
        g.adj_set("v", nb, v[nb - 1])
        g.adj_set("lam", nb, lam[nb - 1])
    g.rhs_invis_tangent()
    g.rhs_invis_adjoint(fold=False)
    jv = [g.adj_get("rdot", nb) for nb in range(1, case.nblocks + 1)]
    jtl = [g.adj_get("qbar", nb) for nb in range(1, case.nblocks + 1)]
    a = dot(case, lam, jv, ghosts=False)
    b = dot(case, jtl, v, ghosts=True)
    scale = norm(case, lam, False) * norm(case, jv, False)
    print(f"{name}: <lam, J v> {a:.15e}  <J^T lam, v> {b:.15e}  rel {abs(a - b) / scale:.2e}")
    assert abs(a - b) <= 1e-12 * scale


def taylor_errors(g, case, base, v, jv, refill, lam=None, qbar=None, steps=(1e-4, 1e-5, 1e-6, 1e-7)):
    """Central-difference discrepancies at decreasing steps: max-norm of
    (r(q + e v) - r(q - e v)) / 2e - J v relative to |J v| (or, with lam and
    qbar, of <lam, FD> - <qbar, v> relative to |lam| |FD|).  They fall as e^2
    while the tangent is exact (the nonlinear weights, 1 / (1e-6 + IS)^2,
    make the second-order term large at the larger steps), then reach the
    round-off floor."""
    out = []
    for eps in steps:
        plus = [[p[m] + eps * v[nb][m] if m < 5 else p[m] for m in range(6)] for nb, p in enumerate(base)]
        minus = [[p[m] - eps * v[nb][m] if m < 5 else p[m] for m in range(6)] for nb, p in enumerate(base)]
        rp = residual(g, case, plus, refill)
        rm = residual(g, case, minus, refill)
        fd = [[(rp[nb][m] - rm[nb][m]) / (2 * eps) for m in range(5)] for nb in range(case.nblocks)]
        if lam is None:
            num = max(float(np.max(np.abs(interior(fd[nb][m] - jv[nb][m], d))))
                      for nb, d in enumerate(case.dims) for m in range(5))
            den = max(float(np.max(np.abs(interior(jv[nb][m], d)))) for nb, d in enumerate(case.dims) for m in range(5))
            out.append(num / den)
        else:
            a, b = dot(case, lam, fd, False), dot(case, qbar, v, False)
            out.append(abs(a - b) / (norm(case, lam, False) * norm(case, fd, False)))
    return out


@pytest.mark.parametrize("name", CASES)
def test_tangent_matches_central_differences(name):
    case = make(name)
    g = ctx(case)
    base = [g.get_prim(nb) for nb in range(1, case.nblocks + 1)]
    rng = np.random.default_rng(5)
    sc = [max(s, 0.1) for s in state_scales(g, case)]
    v = rand_fields(case, rng, ghosts=True, scale=sc)
    for nb in range(1, case.nblocks + 1):
        g.adj_set("v", nb, v[nb - 1])
    g.rhs_invis_tangent()
    jv = [g.adj_get("rdot", nb) for nb in range(1, case.nblocks + 1)]
    e = taylor_errors(g, case, base, v, jv, refill=False)
    print(f"{name}: tangent vs central differences at steps 1e-4..1e-7:", " ".join(f"{x:.2e}" for x in e))
    # second order in the asymptotic range (the discrepancy falls 100x a decade)
    assert e[-2] / e[-1] > 50 and e[-1] < 1e-4, e


def test_folded_adjoint_on_periodic_box_matches_differences():
    """All ghosts of the periodic box are interface copies, so the folded
    adjoint is the adjoint of the residual with the ghosts refilled."""
    case = make("periodic")
    g = ctx(case)
    base = [g.get_prim(nb) for nb in range(1, case.nblocks + 1)]
    rng = np.random.default_rng(3)
    sc = [max(s, 0.1) for s in state_scales(g, case)]
    v = rand_fields(case, rng, ghosts=False, scale=sc)
    lam = rand_fields(case, rng, ghosts=False)
    g.adj_set("lam", 1, lam[0])
    g.rhs_invis_adjoint(fold=True)
    qbar = [g.adj_get("qbar", 1)]
    e = taylor_errors(g, case, base, v, None, refill=True, lam=lam, qbar=qbar)
    print("periodic box, folded adjoint vs central differences at steps 1e-4..1e-7:", " ".join(f"{x:.2e}" for x in e))
    assert e[-2] / e[-1] > 50 and e[-1] < 1e-7, e


@pytest.mark.parametrize("name", ["vortex_sw", "plate_euler", "box_roe"])
def test_lusgs_operator_transpose(name):
    case = make(name)
    g = ctx(case, phases=True)
    rng = np.random.default_rng(8)
    b = rand_fields(case, rng, ghosts=False)
    y = rand_fields(case, rng, ghosts=False)
    for nb in range(1, case.nblocks + 1):
        g.adj_set("b", nb, b[nb - 1])
    g.lusgs_operator(transpose=False)
    pb = [g.adj_get("x", nb) for nb in range(1, case.nblocks + 1)]
    for nb in range(1, case.nblocks + 1):
        g.adj_set("b", nb, y[nb - 1])
    g.lusgs_operator(transpose=True)
    pty = [g.adj_get("x", nb) for nb in range(1, case.nblocks + 1)]
    a, c = dot(case, y, pb, False), dot(case, pty, b, False)
    scale = norm(case, y, False) * norm(case, pb, False)
    print(f"{name}: <y, P b> {a:.15e}  <P^T y, b> {c:.15e}  rel {abs(a - c) / scale:.2e}")
    assert abs(a - c) <= 1e-12 * scale


def _mxdq(prim, nvec, dq, rad, npn, gama):
    """mxdq_std (LHS.f90:756-828) with gettmhmgm_ns, restated in NumPy."""
    rm, um, vm, wm, pm = prim
    c2 = gama * pm / rm
    cm = np.sqrt(c2)
    v2 = um * um + vm * vm + wm * wm
    hm = gama / (gama - 1.0) * pm / rm + 0.5 * v2
    ct = nvec[0] * um + nvec[1] * vm + nvec[2] * wm
    cgm = max(np.sqrt(nvec[0] ** 2 + nvec[1] ** 2 + nvec[2] ** 2), 1e-30)
    l1 = 0.5 * (ct + npn * rad)
    l4 = 0.5 * (ct + cm * cgm + npn * rad)
    l5 = 0.5 * (ct - cm * cgm + npn * rad)
    x1 = (2.0 * l1 - l4 - l5) / (2.0 * c2)
    x2 = (l4 - l5) / (2.0 * cm)
    nx, ny, nz = nvec[0] / cgm, nvec[1] / cgm, nvec[2] / cgm
    ct = ct / cgm
    ae = gama - 1.0
    dc = ct * dq[0] - nx * dq[1] - ny * dq[2] - nz * dq[3]
    dh = 0.5 * ae * v2 * dq[0] - ae * (um * dq[1] + vm * dq[2] + wm * dq[3] - dq[4])
    c2dc = c2 * dc
    return np.array([l1 * dq[0] - dh * x1 - dc * x2,
                     l1 * dq[1] + (nx * c2dc - um * dh) * x1 + (nx * dh - um * dc) * x2,
                     l1 * dq[2] + (ny * c2dc - vm * dh) * x1 + (ny * dh - vm * dc) * x2,
                     l1 * dq[3] + (nz * c2dc - wm * dh) * x1 + (nz * dh - wm * dc) * x2,
                     l1 * dq[4] + (ct * c2dc - hm * dh) * x1 + (ct * dh - hm * dc) * x2])


def test_lusgs_operator_against_numpy():
    """P b = one lusgs_l and one lusgs_u sweep over the interior, restated
    point by point (neighbours inside the block only)."""
    case = cases.vortex_case(ni=13, nj=9, nk=7, nscheme=4, nflux=1, nsteps=1)
    g = ctx(case, phases=True)
    (ni, nj, nk), gama = case.dims[0], case.params.gama if hasattr(case.params, "gama") else 1.4
    I = lambda a: interior(a, (ni, nj, nk))  # noqa: E731  [k, j, i] of points 1..n
    prim = np.stack([I(g.get(f, 1)) for f in ("r", "u", "v", "w", "p")])
    met = [np.stack([I(g.get(f, 1)) for f in names]) for names in
           (("kcx", "kcy", "kcz"), ("etx", "ety", "etz"), ("ctx", "cty", "ctz"))]
    rad = [I(g.get(f, 1)) for f in ("sra", "srb", "src")]
    coed = 1.0 / (1.0 / I(g.get("dtdt", 1)) + rad[0] + rad[1] + rad[2])
    rng = np.random.default_rng(4)
    b = rand_fields(case, rng, ghosts=False)
    g.adj_set("b", 1, b[0])
    g.lusgs_operator(transpose=False)
    got = np.stack([I(a) for a in g.adj_get("x", 1)])
    bb = np.stack([I(a) for a in b[0]])
    x = np.zeros_like(bb)
    pts = sorted(((i + j + k, k, j, i) for k in range(nk) for j in range(nj) for i in range(ni)))
    for _, k, j, i in pts:  # lusgs_l
        acc = np.zeros(5)
        for d, (dk, dj, di) in enumerate(((0, 0, 1), (0, 1, 0), (1, 0, 0))):
            kk, jj, ii = k - dk, j - dj, i - di
            if min(kk, jj, ii) < 0:
                continue
            acc += _mxdq(prim[:, kk, jj, ii], met[d][:, kk, jj, ii], x[:, kk, jj, ii], rad[d][kk, jj, ii], 1.0, gama)
        x[:, k, j, i] = (-bb[:, k, j, i] + acc) * coed[k, j, i]
    n = (nk, nj, ni)
    for _, k, j, i in reversed(pts):  # lusgs_u
        acc = np.zeros(5)
        for d, (dk, dj, di) in enumerate(((0, 0, 1), (0, 1, 0), (1, 0, 0))):
            kk, jj, ii = k + dk, j + dj, i + di
            if kk >= n[0] or jj >= n[1] or ii >= n[2]:
                continue
            acc += _mxdq(prim[:, kk, jj, ii], met[d][:, kk, jj, ii], x[:, kk, jj, ii], rad[d][kk, jj, ii], -1.0, gama)
        x[:, k, j, i] = x[:, k, j, i] - acc * coed[k, j, i]
    err = float(np.max(np.abs(got - x)) / np.max(np.abs(x)))
    print(f"LU-SGS operator against the NumPy restatement: max rel {err:.2e}")
    assert err < 1e-12


def _face_mask(case, name):
    """1 at the interior points whose dq the step keeps, 0 on physical faces."""
    ni, nj, nk = case.dims[0]
    keep = np.ones((nk, nj, ni))
    if name != "periodic":  # every face of the supersonic box is a physical boundary
        keep[:] = 0.0
        keep[1:-1, 1:-1, 1:-1] = 1.0
    return keep


def _conserved_adjoint(g, case, qbar_int):
    r, u, v, w = (interior(g.get(f, 1), case.dims[0]) for f in ("r", "u", "v", "w"))
    g1, qb = 1.4 - 1.0, qbar_int
    return [qb[0] - (u * qb[1] + v * qb[2] + w * qb[3]) / r + 0.5 * g1 * (u * u + v * v + w * w) * qb[4],
            qb[1] / r - g1 * u * qb[4], qb[2] / r - g1 * v * qb[4], qb[3] / r - g1 * w * qb[4], g1 * qb[4]]


@pytest.mark.parametrize("name", ["box_roe", "periodic"])
def test_adjoint_iteration_is_its_formula(name):
    """Two steps of psi <- psi + Z P^T Z (r_Q^T psi + g) from psi = 0 against
    the same formula assembled from separate calls (the adjoint of the
    residual, the conserved-variable transform, the transposed LU-SGS
    operator, the face mask Z), and the reported norms.  (The fixed point
    itself is not reached on these cases: the linearised step of one
    LU-SGS pair with frozen boundary ghosts and without the interface
    averaging grows slowly.)"""
    case = make(name)
    d = case.dims[0]
    keep = _face_mask(case, name)
    rng = np.random.default_rng(9)
    gobj = rand_fields(case, rng, ghosts=False)[0]
    gi = [interior(a, d) for a in gobj]

    def full(ints):  # interior arrays -> ghosted arrays
        out = []
        for a in ints:
            b = np.zeros((d[2] + 6, d[1] + 6, d[0] + 6))
            b[3:3 + d[2], 3:3 + d[1], 3:3 + d[0]] = a
            out.append(b)
        return out

    def pt(g, t_int):  # Z P^T Z t
        g.adj_set("b", 1, full([a * keep for a in t_int]))
        g.lusgs_operator(transpose=True)
        return [interior(a, d) * keep for a in g.adj_get("x", 1)]

    # the iteration: two steps
    g = ctx(case, phases=True)
    g.adj_set("g", 1, gobj)
    g.adj_zero("psi")
    h1 = g.adjoint_iterate(1)
    psi1 = [interior(a, d) for a in g.adj_get("psi", 1)]
    h2 = g.adjoint_iterate(1)
    psi2 = [interior(a, d) for a in g.adj_get("psi", 1)]
    # the formula from separate calls on a second context
    c = ctx(case, phases=True)
    want1 = pt(c, gi)
    assert abs(h1[0] - np.sqrt(sum(float(np.sum((a * keep) ** 2)) for a in gi))) <= 1e-12 * h1[0]
    c.adj_set("lam", 1, full(want1))
    c.rhs_invis_adjoint(fold=True)
    t = [a + b for a, b in zip(_conserved_adjoint(c, case, [interior(x, d) for x in c.adj_get("qbar", 1)]), gi)]
    want2 = [a + b for a, b in zip(want1, pt(c, t))]
    n2 = np.sqrt(sum(float(np.sum((a * keep) ** 2)) for a in t))
    e1 = max(float(np.max(np.abs(a - b))) for a, b in zip(psi1, want1)) / max(float(np.max(np.abs(a))) for a in want1)
    e2 = max(float(np.max(np.abs(a - b))) for a, b in zip(psi2, want2)) / max(float(np.max(np.abs(a))) for a in want2)
    print(f"{name}: step 1 rel {e1:.2e}, step 2 rel {e2:.2e}, norms {h1[0]:.6e} {h2[0]:.6e} (separate {n2:.6e})")
    assert e1 < 1e-12 and e2 < 1e-11
    assert abs(h2[0] - n2) <= 1e-10 * n2


def test_adjoint_cost_against_primal_residual():
    """Device time of one adjoint evaluation against one primal inviscid
    residual on the vortex (65 x 33 x 17, Steger-Warming); printed, bounded
    loosely (the adjoint recomputes the forward line and carries the flux
    Jacobian and the weights' derivatives)."""
    import time
    case = cases.vortex_case(nscheme=4, nflux=1, nsteps=1)
    g = ctx(case, phases=True)
    rng = np.random.default_rng(1)
    g.adj_set("lam", 1, rand_fields(case, rng, ghosts=False)[0])
    for _ in range(3):
        g.r_h_s_invis()
        g.rhs_invis_adjoint()
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        g.r_h_s_invis()
    tp = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        g.rhs_invis_adjoint()
    ta = (time.perf_counter() - t0) / reps
    print(f"inviscid residual {tp * 1e3:.3f} ms, its adjoint {ta * 1e3:.3f} ms, ratio {ta / tp:.2f}")
    assert ta / tp < 50


def _gmres_and_fixed_point(name, restart, maxiter, tol):
    """GMRES (wcns_b200.adjoint.solve) for Z r_Q^T Z psi = -Z g with a seeded
    g, its residual recomputed with a fresh application of the operator, and
    the device's fixed-point iteration with the same operators from psi = 0
    for as many applications: (GMRES history, fresh residual, fixed-point
    residual over its start)."""
    from wcns_b200 import adjoint
    case = make(name)
    rng = np.random.default_rng(11)
    gvec = [[rng.standard_normal((nk, nj, ni)) for _ in range(5)] for ni, nj, nk in case.dims]
    g = ctx(case, phases=True)
    psi, hist = adjoint.solve(g, case, gvec, restart=restart, tol=tol, maxiter=maxiter)
    S = adjoint.AdjointSystem(g, case)
    b = S.flatten(gvec) * S.mask
    rel = float(np.linalg.norm(S.apply_a(S.flatten(psi)) + b) / np.linalg.norm(b))
    f = ctx(case, phases=True)
    for nb in range(1, case.nblocks + 1):
        ni, nj, nk = case.dims[nb - 1]
        full = []
        for a in gvec[nb - 1]:
            x = np.zeros((nk + 6, nj + 6, ni + 6))
            x[3:3 + nk, 3:3 + nj, 3:3 + ni] = a
            full.append(x)
        f.adj_set("g", nb, full)
    f.adj_zero("psi")
    h = f.adjoint_iterate(len(hist))
    print(f"{name}: GMRES({restart}) {len(hist)} iterations to {hist[-1]:.2e}, fresh check {rel:.2e}; "
          f"fixed point after {len(hist)} steps {h[-1] / h[0]:.2e} of its start")
    return hist, rel, h[-1] / h[0]


def test_adjoint_solve_by_gmres_converges_where_the_fixed_point_grows():
    """The supersonic box: GMRES reaches 1e-9 (about 340 iterations on the
    B200) while the fixed point grows."""
    hist, rel, fixed = _gmres_and_fixed_point("box_roe", restart=40, maxiter=1500, tol=1e-9)
    assert hist[-1] <= 1e-9 and rel <= 1e-8
    assert fixed > 1.0
