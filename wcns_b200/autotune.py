"""Autotuned launch shapes, cached per configuration.

`tuned(g)` leaves the context `g` running the shape its configuration
was tuned to: the cached shape when one is stored for the configuration and
the context accepts it, otherwise the autotuner's choice (wcns_autotune: the
sweep cluster size and lane mode, and the residual kernels' lines per CTA,
each timed on the context's current state), which is then stored.

The configuration key covers everything a shape's speed depends on: the
block sizes, the viscous / SA model, the scheme and flux, the context flags,
the residual precision, the device (name, compute capability, SM count) and
the library build (size and modification time of the shared object).  The
cache is one JSON file: $WCNS_SHAPE_CACHE, else
~/.cache/wcns_b200/shapes.json.
"""
from __future__ import annotations

import hashlib
import json
import os
import time

from . import _lib


def cache_path() -> str:
    p = os.environ.get("WCNS_SHAPE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "wcns_b200", "shapes.json")


def library_id() -> str:
    try:
        st = os.stat(_lib.LIB_PATH)
        return f"{st.st_size}:{st.st_mtime_ns}"
    except OSError:
        return "none"


def config_key(dims, nvis, nscheme, nflux, sa, flags, precision, device, lib) -> str:
    desc = {"dims": [list(map(int, d)) for d in dims], "nvis": int(nvis), "nscheme": int(nscheme),
            "nflux": int(nflux), "sa": bool(sa), "flags": int(flags), "precision": int(precision),
            "device": str(device), "lib": str(lib)}
    return hashlib.sha256(json.dumps(desc, sort_keys=True).encode()).hexdigest()[:32]


def load_cache(path=None) -> dict:
    path = path or cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def store(key, entry, path=None):
    """Adds one entry; the file is replaced atomically (several processes
    may tune at once: the last writer's entries win)."""
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    d = load_cache(path)
    d[key] = entry
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def key_of(g) -> str:
    p = g.case.params
    return config_key(g.dims, p.nvis, p.nscheme, p.nflux, g.sa_ready, g.flags, g.precision, g.device_name(),
                      library_id())


def tuned(g, reps=3, use_cache=True) -> dict:
    """Applies the configuration's tuned shape to `g`; returns {"shape",
    "source" ("cache" or "tuned"), "tune_s", "phase_ms"}."""
    key = key_of(g)
    if use_cache:
        e = load_cache().get(key)
        if e and "shape" in e:
            try:
                g.set_shape(e["shape"])
                return {"shape": g.shape, "source": "cache", "tune_s": 0.0, "phase_ms": e.get("phase_ms")}
            except Exception:  # not valid for this context any more: tune again
                pass
    t0 = time.perf_counter()
    shape, ms = g.autotune(reps)
    dt = time.perf_counter() - t0
    entry = {"shape": shape, "phase_ms": [round(v, 5) for v in ms], "tuned_at": time.strftime("%Y-%m-%d %H:%M:%S")}
    if use_cache:
        try:
            store(key, entry)
        except OSError:  # a read-only home: the shape still applies to this context
            pass
    return {"shape": shape, "source": "tuned", "tune_s": round(dt, 3), "phase_ms": entry["phase_ms"]}
