"""C-ABI library: loads without a GPU and exports every symbol the header declares."""
import ctypes

from meltpooldg_b200 import _lib


def test_library_exports_header_symbols():
    lib = _lib.load()
    names = _lib.header_symbols()
    assert "mpdg_heat_vmult" in names and "mpdg_heat_time_step" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(_lib.header_symbols()) <= set(_lib._SIGS), set(_lib.header_symbols()) - set(_lib._SIGS)


def test_defaults_match_reference():
    lib = _lib.load()
    p = _lib.SolverParams()
    lib.mpdg_solver_params_default(ctypes.byref(p))
    # linear_solver_data.hpp:40-47
    assert p.max_iterations == 10000 and p.rel_tolerance == 1e-12 and p.abs_tolerance == 1e-20
    s = _lib.StepParams()
    lib.mpdg_step_params_default(ctypes.byref(s))
    # nonlinear_solver_data.hpp:13-19
    assert s.newton_max_iterations == 10
    assert s.newton_residual_tolerance == 1e-9 and s.newton_correction_tolerance == 1e-10


def test_invalid_arguments_rejected_without_gpu():
    lib = _lib.load()
    d = _lib.MeshDesc()
    d.degree = 9  # outside 1..6
    h = ctypes.c_void_p()
    assert lib.mpdg_heat_create(ctypes.byref(d), 0, ctypes.byref(h)) == _lib.ERR_INVALID_ARGUMENT
    assert "degree" in _lib.last_error()
