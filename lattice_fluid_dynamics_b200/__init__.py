"""B200 (sm_100a) D3Q19 wind-tunnel solver: a drop-in for the LBM hot path
of Lattice (MarcosAsh/Lattice_Fluid_Dynamics, simulation/lib/lbm.h).

The product is the C-ABI shared library ``liblattice_lbm.so`` (header
``include/lattice_lbm.h``); this package builds it (``build``), binds it
(``capi``) and provides the geometry generators used by the benchmarks
(``geometry``).
"""
from .capi import (LBM_STORAGE_BF16, LBM_STORAGE_FP16, LBM_STORAGE_FP32,
                   LBM_STORAGE_FP64, Grid, Particles, load)

__all__ = ["Grid", "Particles", "load", "LBM_STORAGE_FP32", "LBM_STORAGE_FP16",
           "LBM_STORAGE_BF16", "LBM_STORAGE_FP64"]
