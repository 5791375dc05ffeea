"""B200-native (sm_100a) WCNS residual and LU-SGS update on multi-block grids.

Public pieces:
  * ``wcns_b200.solver.Wcns`` -- the per-step interface (reference phase names)
    over the C ABI of ``libwcns_b200.so`` (``include/wcns_b200.h``);
  * ``wcns_b200.cases`` -- seeded synthetic workloads (grids, BC records,
    initial fields);
  * ``wcns_b200.build`` -- builds the CUDA library for sm_100a.
"""
from . import cases  # noqa: F401

__all__ = ["cases", "solver", "build"]
