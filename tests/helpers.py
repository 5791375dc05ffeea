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
    """Return {name: max relative error over blocks}."""
    out = {}
    nbs = blocks or range(1, len(orc.dims) + 1)
    for name in names:
        worst = 0.0
        for nb in nbs:
            a, b = gpu.get(name, nb), orc.get(name, nb)
            if region == "interior":
                a, b = interior(a, orc.dims[nb - 1]), interior(b, orc.dims[nb - 1])
            worst = max(worst, rel_err(a, b))
        out[name] = worst
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
