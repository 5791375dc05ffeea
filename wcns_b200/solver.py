"""Host-side mirror of the reference's per-step interface for the WCNS path.

The reference drives its hot path from the Fortran time loop
(``Main.f90:79-127``) through argument-less subroutines acting on module
globals.  :class:`Wcns` keeps the same phase names and order, each one a call
into the C ABI of ``libwcns_b200.so`` (``include/wcns_b200.h``).  Errors the
reference answers with ``stop`` (Roe ``c^2 <= 0``, too many non-physical
points, unknown BC type) raise :class:`WcnsError`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

FIELDS = ["r", "u", "v", "w", "p", "t", "dq1", "dq2", "dq3", "dq4", "dq5", "dtdt", "sra", "srb", "src",
          "srva", "srvb", "srvc", "kcx", "kcy", "kcz", "etx", "ety", "etz", "ctx", "cty", "ctz", "vol",
          "qke", "vist", "dist"]
FID = {n: i for i, n in enumerate(FIELDS)}
FORCE_KEYS = ("cfx", "cfy", "cfz", "cmx", "cmy", "cmz", "cl", "cd", "xcp")


class _DeviceSlice:
    """A device array described by __cuda_array_interface__ (version 3)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None, "stream": None}


class WcnsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check(rc):
    if rc != 0:
        raise WcnsError(rc, _lib.last_error())


FLAG_SWEEP_BY_PLANE = 1  # WCNS_FLAG_SWEEP_BY_PLANE
FLAG_SWEEP_WIDE = 2  # WCNS_FLAG_SWEEP_WIDE


def params_struct(p, flags=0) -> _lib.WcnsParams:
    return _lib.WcnsParams(p.moo, p.attack, p.sideslip, p.reynolds, p.tref, p.twall, p.cfl, p.timedt_rate, p.efix,
                           p.csrv, p.nvis, p.nscheme, p.nflux, flags)


class Wcns:
    """One multi-block case resident on the GPU."""

    def __init__(self, case, flags=0):
        L = _lib.load()
        self.case = case
        self.flags = int(flags)
        self.sa_ready = False
        self.dims = [tuple(int(v) for v in d) for d in case.dims]
        self._prm = params_struct(case.params, flags)
        dims = (C.c_int * (3 * len(self.dims)))(*[v for d in self.dims for v in d])
        keep, ptrs = [], []
        for xyz in case.xyz:
            for a in xyz:
                a = np.ascontiguousarray(a, dtype=np.float64)
                keep.append(a)
                ptrs.append(a.ctypes.data)
        xyz_p = (C.c_void_p * len(ptrs))(*ptrs)
        regs = np.ascontiguousarray(case.regions, dtype=np.int32)
        h = C.c_void_p()
        _check(L.wcns_create(C.byref(self._prm), len(self.dims), dims, xyz_p, regs.shape[0],
                             regs.ctypes.data_as(C.POINTER(C.c_int)), C.byref(h)))
        self.h = h
        self._xyz = (keep, xyz_p)
        if getattr(case, "block_moo", None):
            for nb, m in enumerate(case.block_moo, start=1):
                self.set_block_freestream(nb, m)
        for nb, prim in enumerate(case.prim, start=1):
            self.set_prim(nb, prim)

    def close(self):
        if getattr(self, "h", None):
            _lib.load().wcns_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state -------------------------------------------------------------
    def set_prim(self, nb, prim):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in prim]
        _check(_lib.load().wcns_set_prim(self.h, nb, *[a.ctypes.data for a in arrs]))

    def get(self, name, nb, out=None):
        """Copy one field of block nb (ghosted layout) to host memory."""
        ni, nj, nk = self.dims[nb - 1]
        if out is None:
            out = np.empty((nk + 6, nj + 6, ni + 6))
        elif out.shape != (nk + 6, nj + 6, ni + 6) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("output array has the wrong shape, dtype or layout")
        _check(_lib.load().wcns_get_field(self.h, FID[name], nb, out.ctypes.data))
        return out

    def get_prim(self, nb, out=None):
        """Copy r, u, v, w, p (and T when `out` has six arrays or is None) of
        block nb to host memory with one synchronisation; returns the arrays."""
        ni, nj, nk = self.dims[nb - 1]
        shape = (nk + 6, nj + 6, ni + 6)
        if out is None:
            out = [np.empty(shape) for _ in range(6)]
        if len(out) not in (5, 6):
            raise ValueError("get_prim takes five or six output arrays")
        for a in out:
            if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("output array has the wrong shape, dtype or layout")
        ptrs = [a.ctypes.data for a in out] + ([None] if len(out) == 5 else [])
        _check(_lib.load().wcns_get_prim(self.h, nb, *ptrs))
        return out

    def set_prim_all(self, prims):
        """Set r, u, v, w, p, T of every block (prims[nb-1] = six arrays) with
        one synchronisation.  The arrays must be C-contiguous float64 in the
        ghosted layout; they are used in place."""
        if len(prims) != len(self.dims):
            raise ValueError("one list of six arrays per block")
        ptrs = []
        for nb, arrs in enumerate(prims, start=1):
            ptrs += self._checked(nb, arrs, 6)
        vec = (C.c_void_p * len(ptrs))(*ptrs)
        _check(_lib.load().wcns_set_prim_all(self.h, vec))

    def get_prim_all(self, outs):
        """Copy r, u, v, w, p (and T where a block's list has six arrays) of
        every block into `outs` (outs[nb-1] = five or six arrays) with one
        synchronisation."""
        if len(outs) != len(self.dims):
            raise ValueError("one list of five or six arrays per block")
        ptrs = []
        for nb, arrs in enumerate(outs, start=1):
            if len(arrs) not in (5, 6):
                raise ValueError("five or six arrays per block")
            ptrs += self._checked(nb, arrs, len(arrs)) + ([None] if len(arrs) == 5 else [])
        vec = (C.c_void_p * len(ptrs))(*ptrs)
        _check(_lib.load().wcns_get_prim_all(self.h, vec))
        return outs

    def get_flow(self, outs=None):
        """The interior state of every block in the flow-file layout:
        outs[nb-1] = five or six C-contiguous float64 arrays of shape
        (nk, nj, ni) for r, u, v, w, p (and T); one synchronisation."""
        if outs is None:
            outs = [[np.empty((nk, nj, ni)) for _ in range(6)] for ni, nj, nk in self.dims]
        if len(outs) != len(self.dims):
            raise ValueError("one list of five or six arrays per block")
        ptrs = []
        for (ni, nj, nk), arrs in zip(self.dims, outs):
            if len(arrs) not in (5, 6):
                raise ValueError("five or six arrays per block")
            for a in arrs:
                if a.shape != (nk, nj, ni) or a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError("flow array has the wrong shape, dtype or layout")
            ptrs += [a.ctypes.data for a in arrs] + ([None] if len(arrs) == 5 else [])
        vec = (C.c_void_p * len(ptrs))(*ptrs)
        _check(_lib.load().wcns_get_flow(self.h, vec))
        return outs

    def _checked(self, nb, arrs, n):
        ni, nj, nk = self.dims[nb - 1]
        shape = (nk + 6, nj + 6, ni + 6)
        if len(arrs) != n:
            raise ValueError(f"block {nb}: {n} arrays expected")
        for a in arrs:
            if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError(f"block {nb}: array has the wrong shape, dtype or layout")
        return [a.ctypes.data for a in arrs]

    def _interior_ptrs(self, names, arrays):
        if len(arrays) != len(self.dims):
            raise ValueError("one list of arrays per block")
        fields = (C.c_int * len(names))(*[FID[n] for n in names])
        ptrs = []
        for (ni, nj, nk), arrs in zip(self.dims, arrays):
            if len(arrs) != len(names):
                raise ValueError(f"{len(names)} arrays per block")
            for a in arrs:
                if a is None:
                    ptrs.append(None)
                    continue
                if a.shape != (nk, nj, ni) or a.dtype != np.float64 or not a.flags.c_contiguous:
                    raise ValueError("interior array has the wrong shape, dtype or layout")
                ptrs.append(a.ctypes.data)
        return fields, (C.c_void_p * len(ptrs))(*ptrs)

    def set_interior(self, names, arrays):
        """Set the interior points (flow-file layout, shape (nk, nj, ni)) of
        the named fields of every block: arrays[nb-1][q] is field names[q]
        of block nb (None skips it); ghost points keep their device values."""
        fields, vec = self._interior_ptrs(names, arrays)
        _check(_lib.load().wcns_set_interior(self.h, len(names), fields, vec))

    def get_interior(self, names, arrays=None):
        """Copy the interior points of the named fields of every block into
        `arrays` (allocated when None); returns them."""
        if arrays is None:
            arrays = [[np.empty((nk, nj, ni)) for _ in names] for ni, nj, nk in self.dims]
        fields, vec = self._interior_ptrs(names, arrays)
        _check(_lib.load().wcns_get_interior(self.h, len(names), fields, vec))
        return arrays

    def profile_step(self, cap=64):
        """One whole step enqueued phase by phase with CUDA events between
        the phases: list of (phase name, device ms).  Advances the state."""
        ms = np.zeros(cap)
        names = (C.c_char_p * cap)()
        n = C.c_int(0)
        _check(_lib.load().wcns_profile_step(self.h, cap, ms.ctypes.data, names, C.byref(n)))
        return [(names[q].decode(), float(ms[q])) for q in range(n.value)]

    def device_view(self, name, nb):
        """Block nb's ghosted slice of a field on the device, as an object
        with __cuda_array_interface__ (shape (nk+6, nj+6, ni+6), float64):
        torch.as_tensor(view, device="cuda") aliases the context's memory.
        Call sync() before touching it and synchronise after."""
        ptr, count = C.c_void_p(), C.c_longlong()
        _check(_lib.load().wcns_field_device_ptr(self.h, FID[name], nb, C.byref(ptr), C.byref(count)))
        ni, nj, nk = self.dims[nb - 1]
        if count.value != (nk + 6) * (nj + 6) * (ni + 6):
            raise RuntimeError("unexpected field slice size")
        return _DeviceSlice(int(ptr.value), (nk + 6, nj + 6, ni + 6))

    def set(self, name, nb, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        _check(_lib.load().wcns_set_field(self.h, FID[name], nb, arr.ctypes.data))

    # -- per-step phases, reference names (Main.f90:85-109) -----------------
    def boundary_all(self):
        _check(_lib.load().wcns_boundary_all(self.h))

    def initial_q_dq_c_t(self):
        _check(_lib.load().wcns_initial_q_dq_c_t(self.h))

    def timestep_tgh(self):
        _check(_lib.load().wcns_timestep(self.h))

    def r_h_s_vis(self):
        _check(_lib.load().wcns_rhs_vis(self.h))

    def r_h_s_vis_flux(self):
        """r_h_s_vis without the SA model step (wcns_rhs_vis_flux)."""
        _check(_lib.load().wcns_rhs_vis_flux(self.h))

    def communicate_dq_npp(self):
        _check(_lib.load().wcns_communicate_dq(self.h))

    def r_h_s_invis(self):
        _check(_lib.load().wcns_rhs_invis(self.h))

    def l_h_s_tgh(self):
        _check(_lib.load().wcns_lhs(self.h))

    def communicate_pv_npp(self):
        _check(_lib.load().wcns_communicate_pv(self.h))

    # -- Spalart-Allmaras model (turblence.f90) ----------------------------
    def sa_setup(self, timedt_turb=1.0, kmaxlim=0.0):
        """Model arrays, wall distance (calc_wall_dists_parallel) and init_SA;
        fields "qke", "vist", "dist" become readable and writable."""
        _check(_lib.load().wcns_sa_setup(self.h, self._xyz[1], timedt_turb, kmaxlim))
        self.sa_ready = True

    def turbulence(self):
        """turbulence(nb) for every block (RHS.f90:22)."""
        _check(_lib.load().wcns_turbulence(self.h))

    def residual_curve(self):
        nb = len(self.dims)
        res, rmax, rms = np.zeros(nb), np.zeros(nb), np.zeros(1)
        _check(_lib.load().wcns_residual(self.h, res.ctypes.data, rmax.ctypes.data, rms.ctypes.data))
        return res, rmax, float(rms[0])

    def force(self, sref=1.0, lfref=1.0, xref=0.0, yref=0.0, zref=0.0, nwholefield=1):
        """Wall force and moment coefficients (force, PostProcess.f90:1415-1480):
        dict of cfx, cfy, cfz, cmx, cmy, cmz, cl, cd, xcp."""
        ref = np.array([sref, lfref, xref, yref, zref, nwholefield], dtype=np.float64)
        out = np.zeros(9)
        _check(_lib.load().wcns_forces(self.h, ref.ctypes.data, out.ctypes.data))
        return dict(zip(FORCE_KEYS, out))

    def force_blocks(self, nb0, nb1, sref=1.0, lfref=1.0, xref=0.0, yref=0.0, zref=0.0, nwholefield=1):
        """Force coefficients over the walls of blocks nb0..nb1 (one case of a batch)."""
        ref = np.array([sref, lfref, xref, yref, zref, nwholefield], dtype=np.float64)
        out = np.zeros(9)
        _check(_lib.load().wcns_forces_blocks(self.h, nb0, nb1, ref.ctypes.data, out.ctypes.data))
        return dict(zip(FORCE_KEYS, out))

    def set_block_freestream(self, nb, moo):
        """Block nb's free stream at Mach moo (a case of a batch)."""
        _check(_lib.load().wcns_set_block_freestream(self.h, nb, moo))

    def step(self, nsteps=1, history=True):
        """nsteps whole time steps (Main.f90:79-127) replayed from a CUDA graph."""
        hist = np.zeros(nsteps) if history else None
        _check(_lib.load().wcns_step(self.h, nsteps, hist.ctypes.data if history else None))
        return hist

    def step_async(self, nsteps):
        _check(_lib.load().wcns_step_async(self.h, nsteps))

    def sync(self):
        _check(_lib.load().wcns_sync(self.h))

    @property
    def stream(self) -> int:
        return int(_lib.load().wcns_stream(self.h) or 0)

    def launches_per_step(self) -> int:
        return int(_lib.load().wcns_launches_per_step(self.h))

    def selftest_timeout(self, limit_cycles=1000):
        """The sweeps' bounded wait on an mbarrier nothing completes: raises
        WcnsError (WCNS_ERR_CUDA) as a step does after a sweep timeout."""
        _check(_lib.load().wcns_selftest_timeout(self.h, limit_cycles))

    def sweep_mode(self) -> str:
        """How the LU-SGS sweeps run: "clustered", "plane" or "wide"."""
        return ("clustered", "plane", "wide")[int(_lib.load().wcns_sweep_mode(self.h))]

    def set_precision(self, bits: int):
        """64: the FP64 residual (default); 32: the mixed-precision residual
        (FP32 interpolation, fluxes and viscous arithmetic; FP64 metrics,
        smoothness-indicator denominators, dq accumulation and LU-SGS)."""
        _check(_lib.load().wcns_set_precision(self.h, int(bits)))

    @property
    def precision(self) -> int:
        return int(_lib.load().wcns_get_precision(self.h))

    @property
    def shape(self) -> list:
        """[cluster CTAs of the sweeps (0: wide or by plane), fine lanes,
        inviscid lines per CTA, viscous lines per CTA]."""
        out = np.zeros(4, dtype=np.int32)
        _check(_lib.load().wcns_get_shape(self.h, out.ctypes.data))
        return [int(v) for v in out]

    def device_name(self) -> str:
        buf = C.create_string_buffer(256)
        _check(_lib.load().wcns_device_name(self.h, buf, 256))
        return buf.value.decode()

    def set_shape(self, shape):
        arr = np.ascontiguousarray(shape, dtype=np.int32)
        if arr.shape != (4,):
            raise ValueError("a shape has four entries")
        _check(_lib.load().wcns_set_shape(self.h, arr.ctypes.data))

    def autotune(self, reps=3):
        """Times the candidate shapes on the current state and keeps the
        fastest: (shape, best ms of the LU-SGS, inviscid and viscous phases)."""
        out = np.zeros(4, dtype=np.int32)
        ms = np.zeros(3)
        _check(_lib.load().wcns_autotune(self.h, int(reps), out.ctypes.data, ms.ctypes.data))
        return [int(v) for v in out], [float(v) for v in ms]

    # ---- tangent / adjoint of the inviscid residual, LU-SGS operator pair
    ADJ = {"v": 0, "rdot": 1, "lam": 2, "qbar": 3, "b": 4, "x": 5, "g": 6, "psi": 7, "w": 8}

    def adj_set(self, slot, nb, five):
        ni, nj, nk = self.dims[nb - 1]
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in five]
        if len(arrs) != 5 or any(a.shape != (nk + 6, nj + 6, ni + 6) for a in arrs):
            raise ValueError("five arrays of the block's ghosted shape")
        ptrs = (C.c_void_p * 5)(*[a.ctypes.data for a in arrs])
        _check(_lib.load().wcns_adj_set(self.h, self.ADJ[slot], nb, ptrs))

    def adj_get(self, slot, nb):
        ni, nj, nk = self.dims[nb - 1]
        out = [np.empty((nk + 6, nj + 6, ni + 6)) for _ in range(5)]
        ptrs = (C.c_void_p * 5)(*[a.ctypes.data for a in out])
        _check(_lib.load().wcns_adj_get(self.h, self.ADJ[slot], nb, ptrs))
        return out

    def adj_zero(self, slot):
        _check(_lib.load().wcns_adj_zero(self.h, self.ADJ[slot]))

    def rhs_invis_tangent(self):
        """rdot = (dr/dq) v at the current state (r: the inviscid residual)."""
        _check(_lib.load().wcns_rhs_invis_tangent(self.h))

    def rhs_invis_adjoint(self, fold=True):
        """qbar = (dr/dq)^T lam at the current state; fold: interface ghosts'
        adjoint moved to their partner points."""
        _check(_lib.load().wcns_rhs_invis_adjoint(self.h, 1 if fold else 0))

    def lusgs_operator(self, transpose=False):
        """x = P b (or P^T b): one lower and one upper LU-SGS sweep."""
        _check(_lib.load().wcns_lusgs_operator(self.h, 1 if transpose else 0))

    def adjoint_iterate(self, iters):
        """psi <- psi + P^T (r_Q^T psi + g), iters times; the norms of
        r_Q^T psi + g before each step."""
        hist = np.zeros(int(iters))
        _check(_lib.load().wcns_adjoint_iterate(self.h, int(iters), hist.ctypes.data))
        return hist

    def n_multipoints(self) -> int:
        return int(_lib.load().wcns_n_multipoints(self.h))
