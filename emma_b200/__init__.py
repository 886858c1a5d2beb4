"""emma_b200 -- B200 (sm_100a) hydro level advance for EMMA oct trees.

The product is libemmahydro.so (C ABI, include/emma_hydro.h); this package holds
its ctypes bindings, a host oct-tree builder with EMMA's construction order,
and the synthetic benchmark configurations.
"""
from ._lib import (PREC_FP64, PREC_MIXED, TRANS_XM, TRANS_XP, TRANS_YM, TRANS_YP, TRANS_ZM,  # noqa: F401
                   TRANS_ZP, lib)
from .tree import OctTree  # noqa: F401
from .hydro import ResidentHydro, HydroSolver, advancehydroGPU, clean_new_hydro, CpuInfo, RunParams  # noqa: F401
