"""Synthetic multi-block workloads for the WCNS residual/LU-SGS path.

Each case is the set of inputs the reference's pre-processing produces from a
PLOT3D grid, a 1976-format BC file and a ``param.dat`` namelist
(``PreProcess.f90:2-65``): block dimensions, grid coordinates, BC region
records (the integer content of the BC file, ``parallel.f90:852-929``),
namelist parameters, and the initial primitive field with its 3-deep ghost
frame.  The grids are generated here from seeds; no external data is read.

Field arrays use the reference's ghosted index space ``(-2:n+3)`` in each
direction with i fastest, i.e. numpy shape ``(nk+6, nj+6, ni+6)``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

GAMMA = 1.4
PAI = 3.14159265  # Globalvar.f90:238, used by init_inflow for the angle of attack


@dataclass
class Params:
    """The ``param.dat`` namelist values that the hot path reads."""

    moo: float = 0.5
    attack: float = 0.0
    sideslip: float = 0.0
    reynolds: float = 1.0e5
    tref: float = 288.15
    twall: float = -1.0
    cfl: float = 2.0
    timedt_rate: float = 1.1
    efix: float = 0.1
    csrv: float = 1.0
    nvis: int = 0
    nscheme: int = 4
    nflux: int = 1

    def freestream(self):
        """Non-dimensional free stream of ``init_inflow`` (PreProcess.f90:968-1113)."""
        a = self.attack * PAI / 180.0
        b = self.sideslip * PAI / 180.0
        roo = 1.0
        uoo = math.cos(a) * math.cos(b)
        voo = math.sin(a) * math.cos(b)
        woo = math.sin(b)
        poo = 1.0 / (GAMMA * self.moo * self.moo)
        return roo, uoo, voo, woo, poo


@dataclass
class Case:
    name: str
    params: Params
    dims: list  # [(ni, nj, nk)] per block
    xyz: list  # [(x, y, z)] per block, each shape (nk, nj, ni)
    regions: np.ndarray  # (nregions, 16) int32 BC records
    prim: list = field(default_factory=list)  # [(r,u,v,w,p,t)] ghosted per block
    nsteps: int = 100
    description: str = ""
    # Spalart-Allmaras settings ($step timedt_turb, $turbulence kmaxlim) for
    # nlamtur=1, nameturb='SA' runs; None for laminar/Euler cases
    sa: dict | None = None
    # a batch of independent cases in one context: each block's Mach number
    # (None: params.moo everywhere) and each case's block range (nb0, nb1)
    block_moo: list | None = None
    groups: list | None = None

    @property
    def npoints(self) -> int:
        return int(sum(ni * nj * nk for ni, nj, nk in self.dims))

    @property
    def nblocks(self) -> int:
        return len(self.dims)


# ----------------------------------------------------------------------------
# BC records.  One record = the 16 integers the reference reads for a region:
#   nb, s_st1, s_ed1, s_st2, s_ed2, s_st3, s_ed3, bctype,
#   t_st1, t_ed1, t_st2, t_ed2, t_st3, t_ed3, nbt, ibcwin
# (the t_*/nbt/ibcwin part is zero unless bctype < 0).
# ----------------------------------------------------------------------------

def _face(dims, face):
    """Index ranges of a whole block face: face in {'i-','i+','j-','j+','k-','k+'}."""
    ni, nj, nk = dims
    rng = [[1, ni], [1, nj], [1, nk]]
    d = "ijk".index(face[0])
    v = 1 if face[1] == "-" else dims[d]
    rng[d] = [v, v]
    return rng


class _RegionList:
    def __init__(self):
        self.recs = []  # per block list of records

    def add(self, nb, rng, bctype, trng=None, nbt=0):
        self.recs.append([nb, rng, bctype, trng, nbt])
        return len(self.recs) - 1

    def connect(self, nb, rng, nbt, trng):
        a = self.add(nb, rng, -1, trng, nbt)
        b = self.add(nbt, trng, -1, rng, nb)
        self.recs[a].append(b)
        self.recs[b].append(a)

    def array(self):
        # ibcwin = index of the partner region within its block (1-based), in
        # the order regions are listed per block.
        order = {}
        per_block = {}
        for idx, rec in enumerate(self.recs):
            per_block.setdefault(rec[0], []).append(idx)
        for nb, lst in per_block.items():
            for pos, idx in enumerate(lst):
                order[idx] = pos + 1
        out = []
        for nb in sorted(per_block):
            for idx in per_block[nb]:
                nbb, rng, bctype, trng, nbt = self.recs[idx][:5]
                row = [nbb, rng[0][0], rng[0][1], rng[1][0], rng[1][1], rng[2][0], rng[2][1], bctype]
                if bctype < 0:
                    partner = self.recs[idx][5]
                    row += [trng[0][0], trng[0][1], trng[1][0], trng[1][1], trng[2][0], trng[2][1], nbt, order[partner]]
                else:
                    row += [0] * 8
                out.append(row)
        return np.asarray(out, dtype=np.int32)


def write_bc_file(path, dims, regions, names=None):
    """Write the 1976-format BC file the reference reads (parallel.f90:852-929)."""
    lines = ["    1976", f"{len(dims):8d}", f"{len(dims):8d}"]
    for nb, (ni, nj, nk) in enumerate(dims, start=1):
        lines.append(f"{nb:8d}")
        lines.append(f"{ni:8d}{nj:8d}{nk:8d}")
        lines.append(f" {names[nb - 1] if names else f'blk-{nb}'}")
        recs = regions[regions[:, 0] == nb]
        lines.append(f"{len(recs):8d}")
        for r in recs:
            lines.append("".join(f"{v:8d}" for v in r[1:8]))
            if r[7] < 0:
                lines.append("        " + "".join(f"{v:8d}" for v in r[8:16]))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_bc_file(path):
    """Parse a 1976-format BC file into (dims, regions)."""
    toks = open(path).read().split("\n")
    it = iter([t for t in toks if t.strip()])
    if int(next(it).split()[0]) != 1976:
        raise ValueError("not a 1976-format BC file")
    next(it)
    nblocks = int(next(it).split()[0])
    dims, recs = [], []
    for _ in range(nblocks):
        nb = len(dims) + 1
        next(it)  # pid
        dims.append(tuple(int(v) for v in next(it).split()[:3]))
        next(it)  # block name
        nr = int(next(it).split()[0])
        for _ in range(nr):
            v = [int(x) for x in next(it).split()[:7]]
            row = [nb] + v
            if v[6] < 0:
                row += [int(x) for x in next(it).split()[:8]]
            else:
                row += [0] * 8
            recs.append(row)
    return dims, np.asarray(recs, dtype=np.int32)


# ----------------------------------------------------------------------------
# Field helpers
# ----------------------------------------------------------------------------

def ghosted_uniform(dims, values):
    ni, nj, nk = dims
    return [np.full((nk + 6, nj + 6, ni + 6), v, dtype=np.float64) for v in values]


def interior(a, dims):
    ni, nj, nk = dims
    return a[3:3 + nk, 3:3 + nj, 3:3 + ni]


def freestream_prim(params: Params, dims):
    roo, uoo, voo, woo, poo = params.freestream()
    return ghosted_uniform(dims, (roo, uoo, voo, woo, poo, 1.0))


# ----------------------------------------------------------------------------
# Config 1: isentropic vortex, single periodic block
# ----------------------------------------------------------------------------

def vortex_case(ni=65, nj=33, nk=17, nscheme=4, nflux=1, seed=0, nsteps=100,
                lx=10.0, ly=5.0, lz=2.5, strength=5.0, radius=1.0, noise=1.0e-6) -> Case:
    """Plain FP64 Euler, one block on [0,lx]x[0,ly]x[0,lz], periodic in x and z
    through self-connections (bctype -1, nbt = 1), far field in y.  Isentropic
    vortex (strength 5, radius 1) on a Mach 0.5 free stream plus seeded uniform
    density noise of amplitude 1e-6."""
    prm = Params(moo=0.5, nvis=0, nscheme=nscheme, nflux=nflux, cfl=2.0, timedt_rate=1.1)
    dims = [(ni, nj, nk)]
    x1 = np.linspace(0.0, lx, ni)
    y1 = np.linspace(0.0, ly, nj)
    z1 = np.linspace(0.0, lz, nk)
    z, y, x = np.meshgrid(z1, y1, x1, indexing="ij")
    rl = _RegionList()
    d = dims[0]
    rl.connect(1, _face(d, "i-"), 1, _face(d, "i+"))
    rl.connect(1, _face(d, "k-"), 1, _face(d, "k+"))
    rl.add(1, _face(d, "j-"), 4)
    rl.add(1, _face(d, "j+"), 4)
    regions = rl.array()
    roo, uoo, voo, woo, poo = prm.freestream()
    r, u, v, w, p, t = freestream_prim(prm, d)
    # Shu's vortex in units rho_inf = p_inf = 1, rescaled to this free stream.
    xc, yc = 0.5 * lx, 0.5 * ly
    dx, dy = (x - xc) / radius, (y - yc) / radius
    r2 = dx * dx + dy * dy
    f = np.exp(0.5 * (1.0 - r2))
    du = -strength / (2.0 * math.pi) * f * dy
    dv = strength / (2.0 * math.pi) * f * dx
    tt = 1.0 - (GAMMA - 1.0) * strength ** 2 / (8.0 * GAMMA * math.pi ** 2) * f * f
    rho = tt ** (1.0 / (GAMMA - 1.0))
    cscale = math.sqrt(poo / roo)
    rng = np.random.default_rng(seed)
    rho = rho + rng.uniform(-noise, noise, size=rho.shape)
    interior(r, d)[...] = rho
    interior(u, d)[...] = uoo + du * cscale
    interior(v, d)[...] = voo + dv * cscale
    interior(w, d)[...] = woo
    interior(p, d)[...] = poo * tt ** (GAMMA / (GAMMA - 1.0))
    return Case("vortex", prm, dims, [(x, y, z)], regions, [(r, u, v, w, p, t)], nsteps,
                f"isentropic vortex {ni}x{nj}x{nk}, nscheme={nscheme}, nflux={nflux}")


# ----------------------------------------------------------------------------
# Config 2: laminar flat plate, 8 blocks of uneven sizes
# ----------------------------------------------------------------------------

def _tanh_wall(n, height, first):
    """n points on [0,height] clustered at 0 with first spacing `first`."""
    eta = np.linspace(0.0, 1.0, n)
    lo, hi = 1e-6, 20.0
    for _ in range(200):
        beta = 0.5 * (lo + hi)
        d1 = height * (1.0 - math.tanh(beta * (1.0 - eta[1])) / math.tanh(beta))
        if d1 > first:
            lo = beta
        else:
            hi = beta
    beta = 0.5 * (lo + hi)
    return height * (1.0 - np.tanh(beta * (1.0 - eta)) / math.tanh(beta))


def _geometric(n, y0, y1, first):
    """n points on [y0,y1] with geometric growth starting at spacing `first`."""
    span = y1 - y0
    m = n - 1
    if first * m >= span:
        return np.linspace(y0, y1, n)
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        s = first * (r ** m - 1.0) / (r - 1.0)
        if s > span:
            hi = r
        else:
            lo = r
    r = 0.5 * (lo + hi)
    d = first * r ** np.arange(m)
    y = np.concatenate([[0.0], np.cumsum(d)])
    return y0 + y * (span / y[-1])


def plate_case(a=65, e=33, h1=65, h2=33, hc=49, nk=9, nscheme=41, nflux=3, nsteps=2000,
               first=1.0e-5, cfl=2.0) -> Case:
    """Laminar FP64 Navier-Stokes flat plate, Re_L = 1e5, Mach 0.3.

    Blocks (i along x, j wall-normal, k spanwise), full size:
      1: 129x65x9 (plate, x in [0,0.5])     2: 97x65x9 (plate, x in [0.5,1])
      3: 65x49x9  (above block 4)            4,5: 65x33x9 (above block 1)
      6,7,8: 33x33x9 (above block 2)
    Wall (isothermal at the free-stream temperature) on the j=1 faces of blocks
    1-2, symmetry on every k face, far field on the remaining outer faces,
    one-to-one point-matched interfaces elsewhere.  Wall-normal tanh
    stretching with first spacing `first` (in units of the plate length)."""
    na, nb = 2 * a - 1, 3 * e - 2
    prm = Params(moo=0.3, reynolds=1.0e5, tref=288.15, twall=288.15, nvis=1, nscheme=nscheme,
                 nflux=nflux, cfl=cfl, timedt_rate=1.1, efix=0.1, csrv=1.0)
    y_row1 = _tanh_wall(h1, 0.05, first)
    y_row2 = _geometric(h2, 0.05, 0.25, y_row1[-1] - y_row1[-2])
    y_top = _geometric(hc, 0.25, 1.0, y_row2[-1] - y_row2[-2])
    x_a = np.linspace(0.0, 0.5, na)
    x_b = np.linspace(0.5, 1.0, nb)
    x_row2 = np.concatenate([x_a, x_b[1:]])
    zs = np.linspace(0.0, 0.03, nk)

    blocks = [  # (x coords, y coords)
        (x_a, y_row1), (x_b, y_row1), (x_row2[0:a], y_top),
        (x_row2[0:a], y_row2), (x_row2[a - 1:2 * a - 1], y_row2),
        (x_row2[na - 1:na - 1 + e], y_row2), (x_row2[na + e - 2:na + 2 * e - 2], y_row2),
        (x_row2[na + 2 * e - 3:na + 3 * e - 3], y_row2),
    ]
    dims, xyz = [], []
    for xs, ys in blocks:
        dims.append((len(xs), len(ys), nk))
        z, y, x = np.meshgrid(zs, ys, xs, indexing="ij")
        xyz.append((np.ascontiguousarray(x), np.ascontiguousarray(y), np.ascontiguousarray(z)))
    rl = _RegionList()
    D = {n + 1: d for n, d in enumerate(dims)}

    def rng(nb_, i0, i1, j0, j1, k0=1, k1=None):
        return [[i0, i1], [j0, j1], [k0, k1 if k1 is not None else nk]]

    # block 1 (A)
    rl.add(1, _face(D[1], "i-"), 4)
    rl.add(1, _face(D[1], "j-"), 2)
    rl.connect(1, _face(D[1], "i+"), 2, _face(D[2], "i-"))
    rl.connect(1, rng(1, 1, a, h1, h1), 4, rng(4, 1, a, 1, 1))
    rl.connect(1, rng(1, a, na, h1, h1), 5, rng(5, 1, a, 1, 1))
    # block 2 (B)
    rl.add(2, _face(D[2], "i+"), 4)
    rl.add(2, _face(D[2], "j-"), 2)
    rl.connect(2, rng(2, 1, e, h1, h1), 6, rng(6, 1, e, 1, 1))
    rl.connect(2, rng(2, e, 2 * e - 1, h1, h1), 7, rng(7, 1, e, 1, 1))
    rl.connect(2, rng(2, 2 * e - 1, nb, h1, h1), 8, rng(8, 1, e, 1, 1))
    # block 3 (C) on top of block 4
    rl.connect(3, _face(D[3], "j-"), 4, _face(D[4], "j+"))
    rl.add(3, _face(D[3], "i-"), 4)
    rl.add(3, _face(D[3], "i+"), 4)
    rl.add(3, _face(D[3], "j+"), 4)
    # row 2
    rl.add(4, _face(D[4], "i-"), 4)
    rl.connect(4, _face(D[4], "i+"), 5, _face(D[5], "i-"))
    rl.connect(5, _face(D[5], "i+"), 6, _face(D[6], "i-"))
    rl.add(5, _face(D[5], "j+"), 4)
    rl.connect(6, _face(D[6], "i+"), 7, _face(D[7], "i-"))
    rl.add(6, _face(D[6], "j+"), 4)
    rl.connect(7, _face(D[7], "i+"), 8, _face(D[8], "i-"))
    rl.add(7, _face(D[7], "j+"), 4)
    rl.add(8, _face(D[8], "i+"), 4)
    rl.add(8, _face(D[8], "j+"), 4)
    for nbk in range(1, 9):
        rl.add(nbk, _face(D[nbk], "k-"), 3)
        rl.add(nbk, _face(D[nbk], "k+"), 3)
    regions = rl.array()
    prim = [tuple(freestream_prim(prm, d)) for d in dims]
    return Case("plate", prm, dims, xyz, regions, prim, nsteps,
                f"laminar plate, 8 blocks, {sum(x*y*z for x, y, z in dims)} points")


def small_plate_case(**kw) -> Case:
    """The flat-plate topology at reduced sizes (for CPU-speed tests)."""
    args = dict(a=9, e=7, h1=11, h2=7, hc=7, nk=7, nsteps=20, first=1.0e-3)
    args.update(kw)
    return plate_case(**args)


# ----------------------------------------------------------------------------
# Config 3: turbulent channel with a Gaussian bump, 24 blocks (SA model)
# ----------------------------------------------------------------------------

def _uneven_splits(n, m, rng, spread=0.25):
    """m contiguous ranges of the global indices 0..n-1 that share their end
    points (point-matched interfaces), of seeded uneven length."""
    base = (n - 1) / m
    cuts = [0]
    for b in range(1, m):
        c = int(round(b * base + rng.uniform(-spread, spread) * base))
        cuts.append(min(max(c, cuts[-1] + 4), n - 1 - 4 * (m - b)))
    cuts.append(n - 1)
    return [(cuts[b], cuts[b + 1]) for b in range(m)]


def _tanh_both(n, first):
    """n points on [0,1] clustered symmetrically at both ends, first spacing
    about `first`."""
    eta = np.linspace(-1.0, 1.0, n)
    lo, hi = 1e-6, 30.0
    for _ in range(200):
        beta = 0.5 * (lo + hi)
        y = 0.5 * (1.0 + np.tanh(beta * eta) / math.tanh(beta))
        if y[1] - y[0] > first:
            lo = beta
        else:
            hi = beta
    beta = 0.5 * (lo + hi)
    return 0.5 * (1.0 + np.tanh(beta * eta) / math.tanh(beta))


def channel_case(ni=385, nj=129, nk=81, bx=6, by=2, bz=2, length=6.0, span=1.0, bump=0.05, first=2.0e-6,
                 nscheme=41, nflux=3, seed=0, nsteps=200) -> Case:
    """Turbulent channel of height H = 1 with a Gaussian bump of height
    `bump`*H on the lower wall at mid-length, Re_H = 5e6, Mach 0.6, for the
    Spalart-Allmaras model (nlamtur=1, nameturb='SA', ncmpcor=0; timedt_turb
    and kmaxlim as in the reference's param.dat template, 10 and 30000).

    A global ni x nj x nk grid (x along the channel, y across it with tanh
    clustering at both walls, z spanwise) is cut into bx*by*bz blocks at
    seeded uneven positions, joined by point-matched one-to-one interfaces.
    Adiabatic viscous walls (bctype 2) at y = wall and y = H, far field (4) at
    the inlet and outlet, symmetry (3) on the spanwise faces.  The full size
    (24 blocks) holds about 4.1 M points."""
    prm = Params(moo=0.6, reynolds=5.0e6, tref=288.15, twall=-1.0, nvis=1, nscheme=nscheme, nflux=nflux,
                 cfl=2.0, timedt_rate=1.1, efix=0.1, csrv=1.0)
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, length, ni)
    eta = _tanh_both(nj, first)
    zs = np.linspace(0.0, span, nk)
    sx, sy, sz = _uneven_splits(ni, bx, rng), _uneven_splits(nj, by, rng), _uneven_splits(nk, bz, rng)
    sigma = 0.1 * length
    dims, xyz, ids = [], [], {}
    for iz in range(bz):
        for iy in range(by):
            for ix in range(bx):
                (i0, i1), (j0, j1), (k0, k1) = sx[ix], sy[iy], sz[iz]
                z, e, x = np.meshgrid(zs[k0:k1 + 1], eta[j0:j1 + 1], xs[i0:i1 + 1], indexing="ij")
                yw = bump * np.exp(-((x - 0.5 * length) / sigma) ** 2)
                y = yw + e * (1.0 - yw)
                dims.append((i1 - i0 + 1, j1 - j0 + 1, k1 - k0 + 1))
                xyz.append((np.ascontiguousarray(x), np.ascontiguousarray(y), np.ascontiguousarray(z)))
                ids[(ix, iy, iz)] = len(dims)
    rl = _RegionList()
    for (ix, iy, iz), nb in ids.items():
        d = dims[nb - 1]
        if ix == 0:
            rl.add(nb, _face(d, "i-"), 4)
        else:
            nbt = ids[(ix - 1, iy, iz)]
            rl.connect(nb, _face(d, "i-"), nbt, _face(dims[nbt - 1], "i+"))
        if ix == bx - 1:
            rl.add(nb, _face(d, "i+"), 4)
        if iy == 0:
            rl.add(nb, _face(d, "j-"), 2)
        else:
            nbt = ids[(ix, iy - 1, iz)]
            rl.connect(nb, _face(d, "j-"), nbt, _face(dims[nbt - 1], "j+"))
        if iy == by - 1:
            rl.add(nb, _face(d, "j+"), 2)
        if iz == 0:
            rl.add(nb, _face(d, "k-"), 3)
        else:
            nbt = ids[(ix, iy, iz - 1)]
            rl.connect(nb, _face(d, "k-"), nbt, _face(dims[nbt - 1], "k+"))
        if iz == bz - 1:
            rl.add(nb, _face(d, "k+"), 3)
    regions = rl.array()
    prim = [tuple(freestream_prim(prm, d)) for d in dims]
    npts = sum(a * b * c for a, b, c in dims)
    return Case("channel", prm, dims, xyz, regions, prim, nsteps,
                f"SA channel with bump, {len(dims)} blocks, {npts} points",
                sa={"timedt_turb": 10.0, "kmaxlim": 30000.0})


def small_channel_case(**kw) -> Case:
    """The channel topology (24 blocks) at reduced sizes (for CPU-speed tests)."""
    args = dict(ni=49, nj=25, nk=13, first=1.0e-3, nsteps=10)
    args.update(kw)
    return channel_case(**args)


def batch_case(ncases=64, seed=0, nsteps=50) -> Case:
    """Independent small channel cases with a wall bump, one block each, for
    one batched context: block sizes drawn from 17^3 .. 49x33x17, Mach from
    U[0.3, 0.8], bump height (fraction of the channel height) from
    U[0.02, 0.08], by seed.  The common parameters are those of the SA
    channel (Re_H 5e6, adiabatic walls, far-field inlet and outlet, spanwise
    symmetry); every case keeps its own Mach number through block_moo and its
    blocks (here one) through groups."""
    rng = np.random.default_rng(seed)
    dims, xyz, prim, regs, moo, groups = [], [], [], [], [], []
    first = None
    for c in range(ncases):
        ni, nj, nk = int(rng.integers(17, 50)), int(rng.integers(17, 34)), 17
        m, h = float(rng.uniform(0.3, 0.8)), float(rng.uniform(0.02, 0.08))
        one = channel_case(ni=ni, nj=nj, nk=nk, bx=1, by=1, bz=1, bump=h, first=1.0e-3, seed=seed + c)
        one.params.moo = m
        if first is None:
            first = one
        nb = len(dims) + 1
        dims += one.dims
        xyz += one.xyz
        prim.append(tuple(freestream_prim(one.params, one.dims[0])))
        r = one.regions.copy()
        r[:, 0] += nb - 1
        r[:, 14] = np.where(r[:, 7] < 0, r[:, 14] + nb - 1, r[:, 14])
        regs.append(r)
        moo.append(m)
        groups.append((nb, nb + len(one.dims) - 1))
    npts = sum(a * b * c for a, b, c in dims)
    return Case("batch", first.params, dims, xyz, np.concatenate(regs), prim, nsteps,
                f"{ncases} independent SA bump cases, one block each, {npts} points",
                sa=first.sa, block_moo=moo, groups=groups)


def batch_member(case: Case, q: int) -> Case:
    """Case q of a batch as a case of its own (its blocks, BC records and Mach)."""
    nb0, nb1 = case.groups[q]
    sel = (case.regions[:, 0] >= nb0) & (case.regions[:, 0] <= nb1)
    r = case.regions[sel].copy()
    r[:, 0] -= nb0 - 1
    r[:, 14] = np.where(r[:, 7] < 0, r[:, 14] - (nb0 - 1), r[:, 14])
    prm = Params(**{k: getattr(case.params, k) for k in Params.__dataclass_fields__})
    prm.moo = case.block_moo[nb0 - 1]
    return Case(f"{case.name}_{q}", prm, case.dims[nb0 - 1:nb1], case.xyz[nb0 - 1:nb1], r,
                [tuple(a.copy() for a in p) for p in case.prim[nb0 - 1:nb1]], case.nsteps, "", sa=case.sa)


CASES = {"vortex": vortex_case, "plate": plate_case, "small_plate": small_plate_case,
         "channel": channel_case, "small_channel": small_channel_case, "batch": batch_case}
