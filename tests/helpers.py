"""Shared comparison helpers for the parity tests."""
import numpy as np


def interior(a, dims):
    ni, nj, nk = dims
    return a[3:3 + nk, 3:3 + nj, 3:3 + ni]


def rel_err(a, b):
    """max |a-b| / max |b| (0 when both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.max(np.abs(a - b)) if a.size else 0.0
    s = np.max(np.abs(b)) if b.size else 0.0
    if d == 0.0:
        return 0.0
    return d / s if s > 0 else np.inf


def compare_fields(gpu, orc, names, blocks=None, region="interior"):
    """Return {name: max |gpu - oracle| over all blocks / max |oracle| over
    all blocks}.  The scale is the field's magnitude over the whole case: in
    a block where a residual component is tiny (nearly uniform flow) its
    values are the cancellation of O(1) fluxes and carry round-off at the
    case's scale, not at their own."""
    out = {}
    nbs = blocks or range(1, len(orc.dims) + 1)
    for name in names:
        num, den = 0.0, 0.0
        for nb in nbs:
            a, b = gpu.get(name, nb), orc.get(name, nb)
            if region == "interior":
                a, b = interior(a, orc.dims[nb - 1]), interior(b, orc.dims[nb - 1])
            num = max(num, float(np.max(np.abs(a - b))) if a.size else 0.0)
            den = max(den, float(np.max(np.abs(b))) if b.size else 0.0)
        out[name] = 0.0 if num == 0.0 else (num / den if den > 0 else np.inf)
    return out


def compare_prim_scaled(gpu, orc, blocks=None):
    """Errors of r, u, v, w, p after many steps, each relative to the scale of
    its quantity: density and pressure to their own maxima, every velocity
    component to the maximum speed (a component that is zero by symmetry has
    no scale of its own)."""
    nbs = blocks or range(1, len(orc.dims) + 1)
    out = {}
    vmax = 0.0
    for nb in nbs:
        d = orc.dims[nb - 1]
        u, v, w = (interior(orc.get(n, nb), d) for n in ("u", "v", "w"))
        vmax = max(vmax, float(np.max(np.sqrt(u * u + v * v + w * w))))
    for name in ("r", "u", "v", "w", "p"):
        num, den = 0.0, 0.0
        for nb in nbs:
            d = orc.dims[nb - 1]
            a, b = interior(gpu.get(name, nb), d), interior(orc.get(name, nb), d)
            num = max(num, float(np.max(np.abs(a - b))))
            den = max(den, float(np.max(np.abs(b))))
        out[name] = num / (vmax if name in ("u", "v", "w") else den) if num else 0.0
    return out


def supersonic_box_case(ni=25, nj=13, nk=9, nscheme=41, nflux=3, seed=3):
    """One Euler block in a Mach-2 stream: supersonic inflow (bctype 5) at
    i-, supersonic outflow (6) at i+, far field (4) at the j faces, symmetry
    (3) at the k faces, and a seeded smooth density bump in the interior so
    that every boundary sees a non-uniform state."""
    from wcns_b200 import cases
    prm = cases.Params(moo=2.0, nvis=0, nscheme=nscheme, nflux=nflux, cfl=1.0, timedt_rate=1.1)
    dims = (ni, nj, nk)
    s = np.linspace(0.0, 1.0, ni)
    t = np.linspace(0.0, 1.0, nj)
    u = np.linspace(0.0, 1.0, nk)
    zz, yy, xx = np.meshgrid(u, t, s, indexing="ij")
    x = 2.0 * xx + 0.03 * np.sin(np.pi * yy)
    y = 1.0 * yy + 0.02 * np.sin(2.0 * np.pi * xx)
    z = 0.5 * zz
    rl = cases._RegionList()
    rl.add(1, cases._face(dims, "i-"), 5)
    rl.add(1, cases._face(dims, "i+"), 6)
    rl.add(1, cases._face(dims, "j-"), 4)
    rl.add(1, cases._face(dims, "j+"), 4)
    rl.add(1, cases._face(dims, "k-"), 3)
    rl.add(1, cases._face(dims, "k+"), 3)
    r, uu, vv, ww, p, tt = cases.freestream_prim(prm, dims)
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0.8, 1.2), rng.uniform(0.4, 0.6)
    bump = 0.2 * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / 0.05)
    cases.interior(r, dims)[...] = 1.0 + bump
    cases.interior(p, dims)[...] = cases.interior(p, dims) * (1.0 + 0.5 * bump)
    return cases.Case("supersonic_box", prm, [dims], [(x, y, z)], rl.array(), [(r, uu, vv, ww, p, tt)], 20,
                      "Mach-2 box with inflow/outflow")


def with_params(case, **kw):
    for k, v in kw.items():
        setattr(case.params, k, v)
    return case


def perturbed(case, amp=0.05, seed=5):
    """Adds a seeded smooth 3-D density/pressure bump to every block's
    interior, so that a case whose free stream is an exact solution (e.g. an
    inviscid plate) still evolves in all three directions."""
    from wcns_b200 import cases
    rng = np.random.default_rng(seed)
    cx, cy = rng.uniform(0.3, 0.7), rng.uniform(0.02, 0.1)
    for nb, d in enumerate(case.dims):
        x, y, z = case.xyz[nb]
        zspan = max(float(np.abs(z).max()), 1e-30)
        bump = amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / 0.02) * (1.0 + 0.5 * np.cos(np.pi * z / zspan))
        r, u, v, w, p, t = case.prim[nb]
        cases.interior(r, d)[...] = cases.interior(r, d) * (1.0 + bump)
        cases.interior(p, d)[...] = cases.interior(p, d) * (1.0 + 1.4 * bump)
    return case


GAMMA = 1.4


def conserved(get, nb, dims):
    """Conserved variables (rho, rho u, rho v, rho w, e) at the interior
    points of block nb from its primitive fields (prim_to_q, Sub1.f90:106)."""
    r, u, v, w, p = (interior(get(n, nb), dims) for n in ("r", "u", "v", "w", "p"))
    return [r, r * u, r * v, r * w, p / (GAMMA - 1.0) + 0.5 * r * (u * u + v * v + w * w)]


def compare_conserved(gpu, orc, blocks=None):
    """max |gpu - oracle| of each conserved variable over all blocks, relative
    to the variable's maximum magnitude over the case; the three momentum
    components share the scale of the momentum magnitude (a component that
    vanishes by symmetry has no scale of its own)."""
    nbs = blocks or range(1, len(orc.dims) + 1)
    num = [0.0] * 5
    den = [0.0] * 5
    mom = 0.0
    for nb in nbs:
        d = orc.dims[nb - 1]
        a, b = conserved(gpu.get, nb, d), conserved(orc.get, nb, d)
        for m in range(5):
            num[m] = max(num[m], float(np.max(np.abs(a[m] - b[m]))))
            den[m] = max(den[m], float(np.max(np.abs(b[m]))))
        mom = max(mom, float(np.max(np.sqrt(b[1] ** 2 + b[2] ** 2 + b[3] ** 2))))
    names = ("rho", "rho_u", "rho_v", "rho_w", "e")
    return {n: (num[m] / (mom if m in (1, 2, 3) else den[m]) if num[m] else 0.0) for m, n in enumerate(names)}


def residual_block_errors(gpu, orc):
    """Relative difference of the per-block residual L2 (residual_curve), its
    maximum and the RMS over all blocks."""
    rg, ro = gpu.residual_curve(), orc.residual()
    res = float(np.max(np.abs(rg[0] - ro[0]) / np.abs(ro[0])))
    rmax = float(np.max(np.abs(rg[1] - ro[1]) / np.abs(ro[1])))
    rms = abs(rg[2] - ro[2]) / abs(ro[2])
    return {"res_l2_per_block": res, "resmax_per_block": rmax, "rms": rms}
