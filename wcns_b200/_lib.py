"""ctypes binding of libwcns_b200.so (the C ABI declared in include/wcns_b200.h).

Loading fails loudly: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwcns_b200.so")


class WcnsParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("moo", "attack", "sideslip", "reynolds", "tref", "twall", "cfl",
                                          "timedt_rate", "efix", "csrv")] + \
               [(n, C.c_int) for n in ("nvis", "nscheme", "nflux", "flags")]


# exported symbols and their signatures (must match include/wcns_b200.h)
_VP = C.c_void_p
SIGNATURES = {
    "wcns_create": (C.c_int, [C.POINTER(WcnsParams), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.c_int,
                              C.POINTER(C.c_int), C.POINTER(C.c_void_p)]),
    "wcns_destroy": (None, [_VP]),
    "wcns_last_error": (C.c_char_p, []),
    "wcns_set_prim": (C.c_int, [_VP, C.c_int] + [_VP] * 6),
    "wcns_get_field": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "wcns_get_prim": (C.c_int, [_VP, C.c_int] + [_VP] * 6),
    "wcns_set_prim_all": (C.c_int, [_VP, C.POINTER(C.c_void_p)]),
    "wcns_get_prim_all": (C.c_int, [_VP, C.POINTER(C.c_void_p)]),
    "wcns_get_flow": (C.c_int, [_VP, C.POINTER(C.c_void_p)]),
    "wcns_set_field": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "wcns_set_interior": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p)]),
    "wcns_get_interior": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p)]),
    "wcns_profile_step": (C.c_int, [_VP, C.c_int, _VP, C.POINTER(C.c_char_p), C.POINTER(C.c_int)]),
    "wcns_boundary_all": (C.c_int, [_VP]),
    "wcns_initial_q_dq_c_t": (C.c_int, [_VP]),
    "wcns_timestep": (C.c_int, [_VP]),
    "wcns_rhs_vis": (C.c_int, [_VP]),
    "wcns_communicate_dq": (C.c_int, [_VP]),
    "wcns_rhs_invis": (C.c_int, [_VP]),
    "wcns_lhs": (C.c_int, [_VP]),
    "wcns_communicate_pv": (C.c_int, [_VP]),
    "wcns_residual": (C.c_int, [_VP, _VP, _VP, _VP]),
    "wcns_step": (C.c_int, [_VP, C.c_int, _VP]),
    "wcns_step_async": (C.c_int, [_VP, C.c_int]),
    "wcns_sync": (C.c_int, [_VP]),
    "wcns_stream": (C.c_void_p, [_VP]),
    "wcns_launches_per_step": (C.c_int, [_VP]),
    "wcns_n_multipoints": (C.c_int, [_VP]),
    "wcns_sweep_mode": (C.c_int, [_VP]),
    "wcns_set_precision": (C.c_int, [_VP, C.c_int]),
    "wcns_get_precision": (C.c_int, [_VP]),
    "wcns_rhs_vis_flux": (C.c_int, [_VP]),
    "wcns_field_device_ptr": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP]),
    "wcns_get_shape": (C.c_int, [_VP, _VP]),
    "wcns_device_name": (C.c_int, [_VP, C.c_char_p, C.c_int]),
    "wcns_set_shape": (C.c_int, [_VP, _VP]),
    "wcns_autotune": (C.c_int, [_VP, C.c_int, _VP, _VP]),
    "wcns_adj_set": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "wcns_adj_get": (C.c_int, [_VP, C.c_int, C.c_int, _VP]),
    "wcns_adj_zero": (C.c_int, [_VP, C.c_int]),
    "wcns_rhs_invis_tangent": (C.c_int, [_VP]),
    "wcns_rhs_invis_adjoint": (C.c_int, [_VP, C.c_int]),
    "wcns_lusgs_operator": (C.c_int, [_VP, C.c_int]),
    "wcns_adjoint_iterate": (C.c_int, [_VP, C.c_int, _VP]),
    "wcns_selftest_timeout": (C.c_int, [_VP, C.c_longlong]),
    "wcns_forces": (C.c_int, [_VP, _VP, _VP]),
    "wcns_forces_blocks": (C.c_int, [_VP, C.c_int, C.c_int, _VP, _VP]),
    "wcns_set_block_freestream": (C.c_int, [_VP, C.c_int, C.c_double]),
    "wcns_sa_setup": (C.c_int, [_VP, C.POINTER(C.c_void_p), C.c_double, C.c_double]),
    "wcns_turbulence": (C.c_int, [_VP]),
    "wcns_residual_noalloc": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_void_p), _VP, _VP, _VP, _VP]),
}

_lib = None


def load():
    """Load the CUDA library; raise if it is missing or cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library {LIB_PATH} is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().wcns_last_error().decode()
