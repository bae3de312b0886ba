"""symphas_b200 -- B200-native explicit finite-difference phase-field solver.

A drop-in for SymPhas's SolverFT path: models keep the MODEL/EVOLUTION
semantics, each model is lowered into one fused sm_100a kernel per step, and
the fields stay resident in HBM.  The compute runs in lib/libsymphas_b200.so
(C ABI in include/symphas_b200.h); this package is the host-side mirror.
"""
from ._capi import SymPhasError, lib
from .model import (BoundaryType, Ensemble, Model, ProblemParameters, SolverFT, Stencil2d2h, Stencil2d4h,
                    Stencil3d2h, ensemble_members, find_solution, model_MA_t, model_MAMK_t, model_MB_t, model_MBMK_t,
                    model_MC_t, model_OP_t)
from .regional import RegionalModel, region_search

__all__ = [
    "BoundaryType", "Ensemble", "Model", "ProblemParameters", "SolverFT", "Stencil2d2h", "Stencil2d4h", "Stencil3d2h",
    "SymPhasError", "ensemble_members", "find_solution", "lib", "model_MA_t", "model_MAMK_t", "model_MB_t",
    "model_MBMK_t", "model_MC_t", "model_OP_t", "RegionalModel", "region_search",
]
