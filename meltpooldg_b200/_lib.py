"""ctypes binding of libmpdg_heat.so (the C ABI declared in include/mpdg_heat.h).

The library is loaded from the package directory; there is no fallback: if the
CUDA library is missing, importing the operator classes raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpdg_heat.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "mpdg_heat.h")

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_MEMORY = 2
ERR_NOT_CONVERGED = 3
ERR_NAN = 4
ERR_BREAKDOWN = 5
ERR_CUDA = 6
ERR_ZERO_TIME_INCREMENT = 7
ERR_NEWTON_NOT_CONVERGED = 8
ERR_NOT_SUPPORTED = 9

LAW_CONSTANT, LAW_LINEAR_K, LAW_LIQUID_SOLID, LAW_GAS_LIQUID, LAW_GAS_LIQUID_SOLID = 0, 1, 2, 3, 4
SOLVER_CG, SOLVER_GMRES = 0, 1
PRECOND_IDENTITY, PRECOND_JACOBI, PRECOND_CHEBYSHEV_JACOBI_F32, PRECOND_MG_F32 = 0, 1, 2, 3
PREDICTOR_NONE, PREDICTOR_LINEAR, PREDICTOR_GIVEN, PREDICTOR_LINEAR_DIRECTION = 0, 1, 2, 3
APPARENT_QLQ, APPARENT_CONSTANT, APPARENT_POLY4_BELL = 0, 1, 2


class MeshDesc(C.Structure):
    _fields_ = [("degree", C.c_int), ("cells", C.c_int * 3), ("lo", C.c_double * 3),
                ("hi", C.c_double * 3), ("perturb", C.c_double), ("seed", C.c_uint64),
                ("dirichlet_mask", C.c_int), ("dirichlet_value", C.c_double * 6)]


class Material(C.Structure):
    _fields_ = [("law", C.c_int), ("sharp", C.c_int), ("volume_specific", C.c_int),
                ("rho_l", C.c_double), ("cp_l", C.c_double), ("k_l", C.c_double),
                ("rho_s", C.c_double), ("cp_s", C.c_double), ("k_s", C.c_double),
                ("T_solidus", C.c_double), ("T_liquidus", C.c_double), ("k1", C.c_double),
                ("sharp_gas_liquid", C.c_int),
                ("rho_g", C.c_double), ("cp_g", C.c_double), ("k_g", C.c_double)]


class SolverParams(C.Structure):
    _fields_ = [("solver", C.c_int), ("preconditioner", C.c_int), ("max_iterations", C.c_int),
                ("rel_tolerance", C.c_double), ("abs_tolerance", C.c_double),
                ("gmres_restart", C.c_int), ("cheb_degree", C.c_int),
                ("cheb_eig_iterations", C.c_int), ("cheb_max_factor", C.c_double),
                ("cheb_min_fraction", C.c_double), ("tol_reference_norm", C.c_double),
                ("cheb_picard", C.c_int), ("cheb_eig_reuse", C.c_int),
                ("mg_smoothing_degree", C.c_int), ("mg_coarse_degree", C.c_int),
                ("mg_smoothing_range", C.c_double), ("mg_min_cells", C.c_int),
                ("mg_fine_pre_steps", C.c_int), ("mg_fine_post_steps", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("true_residual", C.c_double),
                ("lambda_min", C.c_double), ("lambda_max", C.c_double)]


class StepParams(C.Structure):
    _fields_ = [("newton_max_iterations", C.c_int), ("newton_residual_tolerance", C.c_double),
                ("newton_correction_tolerance", C.c_double), ("predictor", C.c_int),
                ("single_linearization", C.c_int), ("linear", SolverParams)]


class StepStats(C.Structure):
    _fields_ = [("newton_iterations", C.c_int), ("linear_iterations", C.c_int),
                ("converged", C.c_int), ("initial_relative_residual", C.c_double),
                ("step_ms", C.c_double)]


LASER_UNIFORM, LASER_GAUSS_VOLUMETRIC, LASER_GAUSS_PROJECTION, LASER_GUSAROV = 0, 1, 2, 3


class Laser(C.Structure):
    _fields_ = [("profile", C.c_int), ("power", C.c_double), ("position", C.c_double * 3),
                ("direction", C.c_double * 3), ("radius", C.c_double),
                ("reflectivity", C.c_double), ("extinction_coefficient", C.c_double),
                ("layer_thickness", C.c_double), ("planar", C.c_int)]


class Counters(C.Structure):
    _fields_ = [("launches", C.c_int64), ("vmult64_calls", C.c_int64),
                ("vmult32_calls", C.c_int64), ("vmult64_ms", C.c_double),
                ("vmult32_ms", C.c_double)]


_P = C.c_void_p
_H = C.c_void_p
_D = C.c_void_p  # device pointers are passed as integers
_SIGS = {
    "mpdg_solver_params_default": (None, [C.POINTER(SolverParams)]),
    "mpdg_step_params_default": (None, [C.POINTER(StepParams)]),
    "mpdg_heat_create": (C.c_int, [C.POINTER(MeshDesc), C.c_int, C.POINTER(_H)]),
    "mpdg_heat_create_slab": (C.c_int, [C.POINTER(MeshDesc), C.c_int, C.c_int, C.c_int,
                                        C.POINTER(_H)]),
    "mpdg_heat_destroy": (C.c_int, [_H]),
    "mpdg_heat_set_stream": (C.c_int, [_H, _P]),
    "mpdg_heat_n_dofs": (C.c_int, [_H, C.POINTER(C.c_int64)]),
    "mpdg_heat_n_cells": (C.c_int, [_H, C.POINTER(C.c_int64)]),
    "mpdg_heat_dof_dims": (C.c_int, [_H, C.POINTER(C.c_int)]),
    "mpdg_heat_device_bytes": (C.c_int, [_H, C.POINTER(C.c_int64)]),
    "mpdg_heat_set_material": (C.c_int, [_H, C.POINTER(Material)]),
    "mpdg_heat_set_fields": (C.c_int, [_H, C.c_void_p, C.c_void_p]),
    "mpdg_heat_reset_time_increment": (C.c_int, [_H, C.c_double]),
    "mpdg_heat_set_boundary": (C.c_int, [_H, C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_double]),
    "mpdg_heat_set_linearization": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_vmult": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_vmult_f32": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_vmult_f32_picard": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_cell_rows_size": (C.c_int, [_H, C.POINTER(C.c_int64)]),
    "mpdg_heat_to_cell_rows_f32": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_vmult_f32_picard_rows": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_picard_cell_rows": (C.c_int, [_H]),
    "mpdg_heat_inverse_diagonal_f32_picard": (C.c_int, [_H, _D]),
    "mpdg_heat_set_picard_tensor_cores": (C.c_int, [_H, C.c_int]),
    "mpdg_heat_picard_tensor_cores": (C.c_int, [_H]),
    "mpdg_picard_tc_matrices": (C.c_int, [_P]),
    "mpdg_heat_compute_inverse_diagonal": (C.c_int, [_H, _D]),
    "mpdg_heat_compute_diagonal": (C.c_int, [_H, _D]),
    "mpdg_heat_create_rhs": (C.c_int, [_H, _D, _D, _D]),
    "mpdg_heat_set_dof_permutation": (C.c_int, [_H, _P]),
    "mpdg_heat_set_laser": (C.c_int, [_H, _P]),
    "mpdg_heat_dcg_start": (C.c_int, [_H, C.c_int64, _D, _D, _D, _D, _D, _D, _D]),
    "mpdg_heat_dcg_dot": (C.c_int, [_H, C.c_int64, _D, _D, _D]),
    "mpdg_heat_dcg_update": (C.c_int, [_H, C.c_int64, _D, _D, _D, _D, _D, _D, _D, _D]),
    "mpdg_heat_dcg_direction": (C.c_int, [_H, _D, _D, _D]),
    "mpdg_heat_invert_diagonal": (C.c_int, [_H, _D]),
    "mpdg_heat_set_linearization_host": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_vmult_host": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_compute_inverse_diagonal_host": (C.c_int, [_H, _D]),
    "mpdg_heat_create_rhs_host": (C.c_int, [_H, _D, _D, _D]),
    "mpdg_heat_distribute_constraints": (C.c_int, [_H, _D]),
    "mpdg_heat_l2_norm": (C.c_int, [_H, _D, C.POINTER(C.c_double)]),
    "mpdg_heat_l2_norm_noalloc": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_support_points": (C.c_int, [_H, _D]),
    "mpdg_heat_laser_source": (C.c_int, [_H, _D, C.POINTER(Laser)]),
    "mpdg_heat_gaussian_source": (C.c_int, [_H, _D, C.c_double, C.POINTER(C.c_double),
                                            C.c_double]),
    "mpdg_heat_preconditioner_update": (C.c_int, [_H]),
    "mpdg_heat_preconditioner_vmult": (C.c_int, [_H, _D, _D]),
    "mpdg_heat_linear_solve": (C.c_int, [_H, C.POINTER(SolverParams), _D, _D,
                                         C.POINTER(SolveStats)]),
    "mpdg_heat_set_guess": (C.c_int, [_H, _D]),
    "mpdg_heat_time_step": (C.c_int, [_H, C.POINTER(StepParams), C.c_double, C.c_double, _D, _D,
                                      _D, C.POINTER(StepStats)]),
    "mpdg_heat_time_step_host": (C.c_int, [_H, C.POINTER(StepParams), C.c_double, C.c_double,
                                           _P, _P, _P, C.POINTER(StepStats)]),
    "mpdg_heat_load_history": (C.c_int, [_H, _P, _P]),
    "mpdg_heat_store_history": (C.c_int, [_H, _P, _P]),
    "mpdg_heat_time_step_resident": (C.c_int, [_H, C.POINTER(StepParams), C.c_double,
                                               C.c_double, _P, _P, C.POINTER(StepStats)]),
    "mpdg_heat_set_timing": (C.c_int, [_H, C.c_int]),
    "mpdg_heat_set_latent_heat": (C.c_int, [_H, C.c_double, C.c_int]),
    "mpdg_heat_set_dirichlet_values": (C.c_int, [_H, _P]),
    "mpdg_material_eval": (C.c_int, [C.POINTER(Material), C.c_double, C.c_int, C.c_double,
                                     C.c_double, _P]),
    "mpdg_amr_create": (C.c_int, [C.POINTER(MeshDesc), _P, C.c_int, C.POINTER(_H)]),
    "mpdg_amr_destroy": (C.c_int, [_H]),
    "mpdg_amr_n_dofs": (C.c_int64, [_H]),
    "mpdg_amr_n_cells": (C.c_int64, [_H]),
    "mpdg_amr_support_points": (C.c_int, [_H, _P]),
    "mpdg_amr_constraint_mask": (C.c_int, [_H, _P]),
    "mpdg_amr_cell_data": (C.c_int, [_H, _P, _P]),
    "mpdg_amr_set_material": (C.c_int, [_H, C.POINTER(Material), C.c_double]),
    "mpdg_amr_vmult": (C.c_int, [_H, _D, _D, _D]),
    "mpdg_amr_inverse_diagonal": (C.c_int, [_H, _D, _D]),
    "mpdg_amr_create_rhs": (C.c_int, [_H, _D, _D, _D, _D]),
    "mpdg_amr_linear_solve": (C.c_int, [_H, _D, _D, _D, C.c_double, C.c_double, C.c_int,
                                         C.POINTER(C.c_int)]),
    "mpdg_amr_time_step": (C.c_int, [_H, C.c_double, C.c_double, _D, _D, _D,
                                      C.POINTER(StepParams), C.POINTER(StepStats)]),
    "mpdg_heat_get_counters": (C.c_int, [_H, C.POINTER(Counters), C.c_int]),
    "mpdg_unet_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(_H)]),
    "mpdg_unet_destroy": (C.c_int, [_H]),
    "mpdg_unet_set_stream": (C.c_int, [_H, _P]),
    "mpdg_unet_n_params": (C.c_int, [_H, C.POINTER(C.c_int64)]),
    "mpdg_unet_dims": (C.c_int, [_H, C.POINTER(C.c_int)]),
    "mpdg_unet_get_params": (C.c_int, [_H, _D]),
    "mpdg_unet_set_params": (C.c_int, [_H, _D]),
    "mpdg_unet_forward": (C.c_int, [_H, _D, _D]),
    "mpdg_unet_backward": (C.c_int, [_H, _D, _D]),
    "mpdg_unet_train_step": (C.c_int, [_H, _D, _D, C.c_float, C.POINTER(C.c_double)]),
    "mpdg_unet_loss": (C.c_int, [_H, _D, C.POINTER(C.c_double)]),
    "mpdg_unet_last_error": (C.c_char_p, []),
    "mpdg_heat_learned_input": (C.c_int, [_H, C.c_int, _D, _D, _D, C.c_double,
                                          C.POINTER(C.c_double), _D]),
    "mpdg_heat_learned_guess": (C.c_int, [_H, _H, C.c_int, _D, _D, _D, C.c_double,
                                          C.c_double, C.c_int, _D, C.POINTER(C.c_double)]),
    "mpdg_heat_learned_direction": (C.c_int, [_H, _H, C.c_int, _D, _D, _D, C.c_double,
                                              C.c_double, _D]),
    "mpdg_heat_set_direction": (C.c_int, [_H, _D]),
    "mpdg_last_error": (C.c_char_p, []),
}

_lock = threading.Lock()
_lib = None


def header_symbols(path: str = HEADER) -> list[str]:
    """Function names declared in the public header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mpdg_[a-z0-9_]+)\s*\(", text)))


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise ImportError(
                    f"{path} not found: build the CUDA library with "
                    "`python -m meltpooldg_b200.build` (there is no CPU fallback)")
            L = C.CDLL(path)
            for name, (res, args) in _SIGS.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    return load().mpdg_last_error().decode(errors="replace")
