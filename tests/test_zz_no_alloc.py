"""wcns_residual_noalloc: the residual norms without any device allocation.

Some callers may not allocate GPU memory when they need the residual -- a
host code whose own pool allocator owns all device memory, or a call made
from inside another library's callback -- so this entry point keeps its
partial sums in a fixed device array of the library and reads the caller's
own device arrays.  It must give exactly what wcns_residual gives for the
same fields (same kernels' arithmetic and reduction order); the bar used here
is the phase tolerance of the parity tests, 1e-12 relative.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one; it also passes alone in a fresh process
(its first call on the device does the one-time set-up).
"""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import rel_err
from wcns_b200 import cases

pytestmark = pytest.mark.gpu

TOL = 1e-12
FIELDS = ["dq1", "dq2", "dq3", "dq4", "dq5", "dtdt", "vol"]


def _noalloc_residual(lib, dims, ptrs):
    nb = len(dims)
    cdims = (C.c_int * (3 * nb))(*[v for d in dims for v in d])
    cptrs = (C.c_void_p * len(ptrs))(*ptrs)
    res, rmax, rms = np.zeros(nb), np.zeros(nb), np.zeros(1)
    rc = lib.wcns_residual_noalloc(nb, cdims, cptrs, res.ctypes.data, rmax.ctypes.data, rms.ctypes.data, None)
    assert rc == 0, lib.wcns_last_error().decode()
    return res, rmax, float(rms[0])


def test_noalloc_residual_matches_wcns_residual():
    import torch

    from wcns_b200 import _lib
    from wcns_b200.solver import Wcns

    lib = _lib.load()
    g = Wcns(cases.small_plate_case())
    # two calls in a row, each on a different state: the second must not be
    # affected by what the first left in the shared scratch array
    for _ in range(2):
        g.step(1)
        res, rmax, rms = g.residual_curve()
        keep, ptrs = [], []
        for nb in range(1, len(g.dims) + 1):
            for name in FIELDS:
                t = torch.from_numpy(g.get(name, nb)).to("cuda")
                keep.append(t)
                ptrs.append(t.data_ptr())
        torch.cuda.synchronize()
        res2, rmax2, rms2 = _noalloc_residual(lib, g.dims, ptrs)
        assert rms > 0.0
        assert rel_err(res2, res) <= TOL
        assert rel_err(rmax2, rmax) <= TOL
        assert abs(rms2 - rms) <= TOL * abs(rms)
    g.close()


def test_noalloc_rejects_too_many_blocks():
    from wcns_b200 import _lib

    lib = _lib.load()
    nb = 257  # WCNS_NOALLOC_MAX_BLOCKS + 1
    cdims = (C.c_int * (3 * nb))(*([5] * (3 * nb)))
    cptrs = (C.c_void_p * (7 * nb))(*([1] * (7 * nb)))
    rc = lib.wcns_residual_noalloc(nb, cdims, cptrs, None, None, None, None)
    assert rc == 1  # WCNS_ERR_ARGUMENT, before any device work
    assert b"maximum" in lib.wcns_last_error()
