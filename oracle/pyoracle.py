"""ctypes wrapper of the CPU oracle (liboracle).  TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check in __graft_entry__.py and the CPU legs of bench.py
may import this module; the product (wcns_b200/) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libwcns_oracle.so")

FIELDS = ["r", "u", "v", "w", "p", "t", "dq1", "dq2", "dq3", "dq4", "dq5", "dtdt", "sra", "srb", "src",
          "srva", "srvb", "srvc", "kcx", "kcy", "kcz", "etx", "ety", "etz", "ctx", "cty", "ctz", "vol",
          "qke", "vist", "dist", "c", "visl", "q1", "q2", "q3", "q4", "q5"]
FID = {n: i for i, n in enumerate(FIELDS)}


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("moo", "attack", "sideslip", "reynolds", "tref", "twall", "cfl",
                                          "timedt_rate", "efix", "csrv")] + \
               [(n, C.c_int) for n in ("nvis", "nscheme", "nflux", "nthreads")]


def build():
    subprocess.run(["make", "-C", HERE, "-s"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p),
                                 C.c_int, C.POINTER(C.c_int)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        for fn in ("orc_boundary_all", "orc_initial_q_dq_c_t", "orc_timestep", "orc_rhs_vis",
                   "orc_communicate_dq", "orc_rhs_invis", "orc_lhs", "orc_communicate_pv", "orc_n_multipoints",
                   "orc_turbulence"):
            getattr(L, fn).argtypes = [C.c_void_p]
            getattr(L, fn).restype = C.c_int
        L.orc_set_prim.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 6
        L.orc_get_field.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.orc_set_field.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.orc_residual.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib = L
    return _lib


def params_struct(p, nthreads=0):
    return OrcParams(p.moo, p.attack, p.sideslip, p.reynolds, p.tref, p.twall, p.cfl, p.timedt_rate, p.efix,
                     p.csrv, p.nvis, p.nscheme, p.nflux, nthreads)


class Oracle:
    """The CPU restatement holding one multi-block case."""

    def __init__(self, case, nthreads=0):
        L = lib()
        self.case = case
        self.dims = [tuple(d) for d in case.dims]
        self._prm = params_struct(case.params, nthreads)
        dims = (C.c_int * (3 * len(self.dims)))(*[v for d in self.dims for v in d])
        self._keep = []
        ptrs = []
        for (x, y, z) in case.xyz:
            for a in (x, y, z):
                a = np.ascontiguousarray(a, dtype=np.float64)
                self._keep.append(a)
                ptrs.append(a.ctypes.data)
        xyz = (C.c_void_p * len(ptrs))(*ptrs)
        regs = np.ascontiguousarray(case.regions, dtype=np.int32)
        self._keep.append(regs)
        self.h = L.orc_create(C.byref(self._prm), len(self.dims), dims, xyz, regs.shape[0],
                              regs.ctypes.data_as(C.POINTER(C.c_int)))
        if not self.h:
            raise RuntimeError("oracle create failed: " + L.orc_last_error().decode())
        for nb, prim in enumerate(case.prim, start=1):
            self.set_prim(nb, prim)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    __del__ = close

    def set_prim(self, nb, prim):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in prim]
        rc = lib().orc_set_prim(self.h, nb, *[a.ctypes.data for a in arrs])
        assert rc == 0

    def get(self, name, nb):
        ni, nj, nk = self.dims[nb - 1]
        out = np.empty((nk + 6, nj + 6, ni + 6))
        rc = lib().orc_get_field(self.h, FID[name], nb, out.ctypes.data)
        assert rc == 0
        return out

    def set(self, name, nb, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        assert lib().orc_set_field(self.h, FID[name], nb, arr.ctypes.data) == 0

    def phase(self, name):
        rc = getattr(lib(), "orc_" + name)(self.h)
        if rc != 0:
            raise RuntimeError(f"oracle {name} failed ({rc}): " + lib().orc_last_error().decode())

    def residual(self):
        nb = len(self.dims)
        res = np.zeros(nb)
        rmax = np.zeros(nb)
        rms = np.zeros(1)
        lib().orc_residual(self.h, res.ctypes.data, rmax.ctypes.data, rms.ctypes.data)
        return res, rmax, float(rms[0])

    def step(self, n=1):
        hist = np.zeros(n)
        rc = lib().orc_step(self.h, n, hist.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"oracle step failed ({rc}): " + lib().orc_last_error().decode())
        return hist

    def force(self, sref=1.0, lfref=1.0, xref=0.0, yref=0.0, zref=0.0, nwholefield=1):
        ref = np.array([sref, lfref, xref, yref, zref, nwholefield], dtype=np.float64)
        out = np.zeros(9)
        L = lib()
        L.orc_forces.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_forces(self.h, ref.ctypes.data, out.ctypes.data)
        return dict(zip(("cfx", "cfy", "cfz", "cmx", "cmy", "cmz", "cl", "cd", "xcp"), out))

    def n_multipoints(self):
        return lib().orc_n_multipoints(self.h)

    def sa_boundary_rules(self, on=True):
        lib().orc_sa_boundary_rules.argtypes = [C.c_void_p, C.c_int]
        assert lib().orc_sa_boundary_rules(self.h, 1 if on else 0) == 0

    def sa_setup(self, timedt_turb=1.0, kmaxlim=0.0, distance=True):
        """init_SA and the model's settings; with distance=False the wall
        distance is not computed (set field "dist" afterwards)."""
        L = lib()
        L.orc_sa_setup_ex.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        assert L.orc_sa_setup_ex(self.h, timedt_turb, kmaxlim, 1 if distance else 0) == 0
