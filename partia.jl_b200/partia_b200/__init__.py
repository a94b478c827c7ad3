"""partia_b200: B200-native SPH interpolation hot path of Partia.jl.

The compute path is the CUDA library libpartia_b200.so (sm_100a) behind the C
ABI declared in include/partia_b200.h; this package is its host-side mirror of
Partia's interpolation API (see api.py) plus a thin context wrapper
(engine.py).
"""
from . import _lib
from ._lib import PsbError, load
from .api import (ArgumentError, B200ComputeBackend, C2_Wendland, C4_Wendland, C6_Wendland, Cartesian,
                  DimensionMismatch, GridBundle, InterpolationCatalog, InterpolationInput, LinearBVH, LinearBVH_,
                  LineSamples, LineSamples_interpolation, M4_spline, M5_spline, M6_spline, PointSamples,
                  PointSamples_interpolation, StructuredGrid, StructuredGrid_interpolation, build_input, flatten,
                  initialize_interpolation, itpGather, itpScatter, itpSymmetric, linrange, matches_lbvh_leaf_order,
                  restore_struct)
from .engine import CatalogC, Context

__all__ = [n for n in dir() if not n.startswith("_")]
