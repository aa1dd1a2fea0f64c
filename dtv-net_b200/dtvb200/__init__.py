"""dtvb200 — B200 cone-beam projector pair and unrolled DTV / FISTA / PDHG updates.

The compute path is the sm_100a kernel library libdtvb200.so behind the C ABI
of include/dtv_b200.h; this package is its host side. There is no CPU path.
"""
from . import _lib, autotune
from ._lib import DtvError
from .geometry import (Geometry, Plan, backward_many, backward_refresh, circular, forward_many,
                       forward_refresh, standard, vector)
from .ops import (BeijingGeometry, BeijingGeometryWithFBP, Projector, RampFilter,
                  StandardGeometry, StandardGeometryWithFBP, fbp_filter, make_functions)
from .tv import diff, diff_abs_sums, l1ball
from .algorithms import ASDPOCS, DTVCP, DTVFISTA, FISTA, Batched, BatchedFISTA, power_norm

__all__ = [
    "DtvError", "Geometry", "Plan", "circular", "standard", "vector", "Projector",
    "StandardGeometry", "StandardGeometryWithFBP", "BeijingGeometry", "BeijingGeometryWithFBP",
    "RampFilter", "fbp_filter", "make_functions", "diff",
    "diff_abs_sums", "l1ball", "DTVCP", "FISTA", "DTVFISTA", "ASDPOCS", "Batched", "BatchedFISTA",
    "power_norm", "forward_many", "backward_many", "forward_refresh", "backward_refresh",
    "library_path",
]


def library_path() -> str:
    return _lib.LIB_PATH
