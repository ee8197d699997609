"""B200-native (sm_100a) implementation of PurineCFD's explicit JST + Spalart-Allmaras
RANS loop, behind the reference's Solver interface (jst-rs/src/solver.rs)."""

from .solver import (DT_GLOBAL, DT_LOCAL, PATH_FUSED, PATH_PASSES, PREC_FP32_SPLIT, PREC_FP64, JstError,
                     NonPhysical, RunReport, Solver)

__all__ = ["Solver", "RunReport", "JstError", "NonPhysical", "PREC_FP64", "PREC_FP32_SPLIT", "DT_GLOBAL",
           "DT_LOCAL", "PATH_FUSED", "PATH_PASSES"]
