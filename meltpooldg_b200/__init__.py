"""B200-native matrix-free heat operator and solve (MeltPoolDG hot path).

The compute path is the CUDA library libmpdg_heat.so (C ABI in
include/mpdg_heat.h); this package is its Python host binding.
"""
from ._lib import (LAW_CONSTANT, LAW_LINEAR_K, LAW_LIQUID_SOLID, PRECOND_CHEBYSHEV_JACOBI_F32,
                   PRECOND_IDENTITY, PRECOND_JACOBI, PREDICTOR_GIVEN, PREDICTOR_LINEAR,
                   PREDICTOR_NONE, SOLVER_CG, SOLVER_GMRES)

__all__ = ["LAW_CONSTANT", "LAW_LINEAR_K", "LAW_LIQUID_SOLID", "PRECOND_CHEBYSHEV_JACOBI_F32",
           "PRECOND_IDENTITY", "PRECOND_JACOBI", "PREDICTOR_GIVEN", "PREDICTOR_LINEAR",
           "PREDICTOR_NONE", "SOLVER_CG", "SOLVER_GMRES"]
