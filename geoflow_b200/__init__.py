"""geoflow_b200 -- B200-native (sm_100a) GeoFLOW spectral-element hot path.

The compute lives in libgfgpu.so (C ABI, include/gfgpu.h); this package is
the Python host-side mirror of the reference interfaces over that ABI.
"""
from . import _abi, gio
from ._abi import GFError, load
from . import workloads
from .ensemble import Ensemble
from .sem import (CGTraits, Context, GBoydFilter, GBurgers, GCG, GGFX, GHelmholtz, GMass,
                  GProjectionFilter, Graph, GridBox, IcosGrid, Problem, filter_matrix, gll_basis)

__all__ = ["GFError", "load", "CGTraits", "Context", "Ensemble", "GBoydFilter", "GBurgers", "GCG", "GGFX",
           "GHelmholtz", "GMass", "GProjectionFilter", "Graph", "GridBox", "IcosGrid", "Problem",
           "filter_matrix", "gll_basis", "_abi", "gio", "workloads"]
