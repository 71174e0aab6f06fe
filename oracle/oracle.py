"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C restatement of MeltPoolDG's matrix-free heat path
(see ``mpdg_oracle.h`` for the reference files it follows). It is the
checker for the CUDA product and the timed CPU baseline; the product never
imports this module. Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
legs of ``bench.py`` use it.

The shared library is compiled on first use for the host it runs on
(``-O3 -march=native -fopenmp``) into ``oracle/_build/<cpu-tag>/``.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "mpdg_oracle.c")
_HDR = os.path.join(_HERE, "mpdg_oracle.h")
_lock = threading.Lock()
_lib = None

LAW_CONSTANT, LAW_LINEAR_K, LAW_LIQUID_SOLID, LAW_GAS_LIQUID, LAW_GAS_LIQUID_SOLID = 0, 1, 2, 3, 4


def _cpu_tag() -> str:
    flags = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = line
                    break
    except OSError:
        pass
    src = open(_SRC, "rb").read() + open(_HDR, "rb").read()
    return hashlib.sha1(flags.encode() + src).hexdigest()[:16]


def build(force: bool = False) -> str:
    """Compile the oracle for this host; returns the library path."""
    out_dir = os.path.join(_HERE, "_build", _cpu_tag())
    so = os.path.join(out_dir, "libmpdg_oracle.so")
    if os.path.exists(so) and not force:
        return so
    os.makedirs(out_dir, exist_ok=True)
    tmp = so + f".tmp{os.getpid()}"
    cmd = ["gcc", "-O3", "-march=native", "-fopenmp", "-fPIC", "-shared", "-std=gnu11",
           "-o", tmp, _SRC, "-lm"]
    subprocess.check_call(cmd)
    os.replace(tmp, so)
    return so


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
                ("rho_g", C.c_double), ("cp_g", C.c_double), ("k_g", C.c_double),
                ("latent_heat", C.c_double), ("apparent_capacity", C.c_int)]


APPARENT_QLQ, APPARENT_CONSTANT, APPARENT_POLY4_BELL = 0, 1, 2


class SolverParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("rel_tolerance", C.c_double),
                ("abs_tolerance", C.c_double), ("precond", C.c_int), ("cheb_degree", C.c_int),
                ("cheb_lambda_min", C.c_double), ("cheb_lambda_max", C.c_double)]


class NewtonParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("residual_tolerance", C.c_double),
                ("correction_tolerance", C.c_double)]


class StepStats(C.Structure):
    _fields_ = [("newton_iterations", C.c_int), ("linear_iterations", C.c_int),
                ("converged", C.c_int)]


_P = C.c_void_p
_D = C.POINTER(C.c_double)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            L = C.CDLL(build())
            L.orc_create.restype = _P
            L.orc_create.argtypes = [C.POINTER(MeshDesc)]
            L.orc_destroy.argtypes = [_P]
            L.orc_n_dofs.restype = C.c_int64
            L.orc_n_dofs.argtypes = [_P]
            L.orc_n_cells.restype = C.c_int64
            L.orc_n_cells.argtypes = [_P]
            L.orc_dof_dims.argtypes = [_P, C.POINTER(C.c_int)]
            L.orc_constraint_mask.argtypes = [_P, C.POINTER(C.c_uint8)]
            L.orc_support_points.argtypes = [_P, _D]
            L.orc_distribute.argtypes = [_P, _D]
            L.orc_set_threads.argtypes = [C.c_int]
            L.orc_set_material.argtypes = [_P, C.POINTER(Material), C.c_double]
            L.orc_set_fields.argtypes = [_P, _D, _D]
            L.orc_material_eval.argtypes = [C.POINTER(Material), C.c_double, C.c_double, _D]
            L.orc_material_eval.restype = None
            L.orc_set_dirichlet_values.argtypes = [_P, _D]
            L.orc_set_dirichlet_values.restype = None
            L.orc_vmult.argtypes = [_P, _D, _D, _D, _D, C.c_int]
            L.orc_inverse_diagonal.argtypes = [_P, _D, _D, _D, C.c_int]
            L.orc_create_rhs.argtypes = [_P, _D, _D, _D, _D]
            L.orc_l2_norm.restype = C.c_double
            L.orc_l2_norm.argtypes = [_P, _D]
            L.orc_cg.restype = C.c_int
            L.orc_cg.argtypes = [_P, C.POINTER(SolverParams), _D, _D, _D, _D, _D, _D]
            L.orc_estimate_eigenvalues.argtypes = [_P, _D, _D, _D, C.c_int, _D, _D]
            L.orc_chebyshev_apply.argtypes = [_P, C.POINTER(SolverParams), _D, _D, _D, _D, _D]
            L.orc_linear_predictor.argtypes = [_P, _D, _D, _D, C.c_double, C.c_double]
            L.orc_time_step_newton.restype = C.c_int
            L.orc_time_step_newton.argtypes = [_P, _D, _D, _D, C.c_double, C.c_double, C.c_int,
                                               C.c_int, C.POINTER(SolverParams), C.POINTER(NewtonParams),
                                               C.POINTER(StepStats)]
            L.orc_gmres.restype = C.c_int
            L.orc_gmres.argtypes = [_P, C.POINTER(SolverParams), C.c_int, _D, _D, _D, _D, _D, _D]
            L.orc_set_boundary.restype = C.c_int
            L.orc_set_boundary.argtypes = [_P, C.c_int, C.c_int, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_double]
            L.orc_gaussian_source.argtypes = [_P, _D, C.c_double, _D, C.c_double]
            L.orc_laser_source.argtypes = [_P, _D, C.c_int, C.c_double, _D, _D, C.c_double,
                                           C.c_double, C.c_double, C.c_double, C.c_int]
            _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def material(law=LAW_CONSTANT, rho=1.0, cp=1.0, k=1.0, k1=0.0, rho_s=None, cp_s=None, k_s=None,
             T_solidus=0.0, T_liquidus=1.0, sharp=False, volume_specific=False, rho_g=None,
             cp_g=None, k_g=None, sharp_gas_liquid=False, latent_heat=0.0,
             apparent_capacity=APPARENT_QLQ) -> Material:
    m = Material()
    m.law = law
    m.sharp = int(sharp)
    m.volume_specific = int(volume_specific)
    m.rho_l, m.cp_l, m.k_l = rho, cp, k
    m.rho_s = rho if rho_s is None else rho_s
    m.cp_s = cp if cp_s is None else cp_s
    m.k_s = k if k_s is None else k_s
    m.T_solidus, m.T_liquidus, m.k1 = T_solidus, T_liquidus, k1
    m.sharp_gas_liquid = int(sharp_gas_liquid)
    m.rho_g = rho if rho_g is None else rho_g
    m.cp_g = cp if cp_g is None else cp_g
    m.k_g = k if k_g is None else k_g
    m.latent_heat = float(latent_heat)
    m.apparent_capacity = int(apparent_capacity)
    return m


def material_eval(m: Material, T: float, H: float = 1.0):
    """(rho*cp, k, d(rho*cp)/dT, dk/dT) of the law at temperature T and heaviside H."""
    out = np.zeros(4)
    lib().orc_material_eval(C.byref(m), float(T), float(H), _ptr(out))
    return tuple(out)


class Oracle:
    """One structured FE_Q(p) box mesh with the oracle operator on it."""

    def __init__(self, degree, cells, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), perturb=0.0,
                 seed=1, dirichlet_mask=0x3F, dirichlet_value=(0.0,) * 6):
        self.L = lib()
        d = MeshDesc()
        d.degree = degree
        for i in range(3):
            d.cells[i] = cells[i]
            d.lo[i] = lo[i]
            d.hi[i] = hi[i]
        d.perturb = perturb
        d.seed = seed
        d.dirichlet_mask = dirichlet_mask
        for i in range(6):
            d.dirichlet_value[i] = dirichlet_value[i]
        self.desc = d
        self.h = self.L.orc_create(C.byref(d))
        if not self.h:
            raise ValueError("invalid mesh description")
        self.n_dofs = int(self.L.orc_n_dofs(self.h))
        self.n_cells = int(self.L.orc_n_cells(self.h))
        dims = (C.c_int * 3)()
        self.L.orc_dof_dims(self.h, dims)
        self.dims = tuple(dims)
        self.degree = degree
        self.dt = 1.0

    def __del__(self):
        try:
            if self.h:
                self.L.orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def mask(self):
        m = np.zeros(self.n_dofs, np.uint8)
        self.L.orc_constraint_mask(self.h, m.ctypes.data_as(C.POINTER(C.c_uint8)))
        return m

    def support_points(self):
        x = np.zeros((self.n_dofs, 3))
        self.L.orc_support_points(self.h, _ptr(x))
        return x

    def distribute(self, u):
        self.L.orc_distribute(self.h, _ptr(u))
        return u

    def set_material(self, m: Material, dt: float):
        rc = self.L.orc_set_material(self.h, C.byref(m), dt)
        if rc != 0:
            raise ValueError("velocity with the linear-k law" if rc == -1 else
                             "apparent capacity with volume-specific rho*cp")
        self.dt = dt
        self._material = m

    def set_dirichlet_values(self, values):
        """Dirichlet values per face (x-, x+, y-, y+, z-, z+) from now on."""
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(6)
        self.L.orc_set_dirichlet_values(self.h, _ptr(v))

    def set_fields(self, heaviside=None, velocity=None):
        """Nodal heaviside (n_dofs) and velocity ((3, n_dofs)) fields; None clears one."""
        H = None if heaviside is None else np.ascontiguousarray(heaviside, np.float64)
        V = None if velocity is None else np.ascontiguousarray(velocity, np.float64).reshape(3, -1)
        self._fields = (H, V)  # the oracle keeps the pointers
        if self.L.orc_set_fields(self.h, _ptr(H), None if V is None else _ptr(V)) != 0:
            raise ValueError("velocity with the linear-k law")

    def set_boundary(self, face, convection=None, radiation=None, neumann=None):
        """convection=(h, T_inf), radiation=(emissivity, T_inf), neumann=q_n."""
        t = (1 if convection else 0) | (2 if radiation else 0) | (4 if neumann is not None else 0)
        hc, tc = convection or (0.0, 0.0)
        e, tr = radiation or (0.0, 0.0)
        rc = self.L.orc_set_boundary(self.h, face, t, hc, tc, e, tr,
                                     0.0 if neumann is None else neumann)
        if rc != 0:
            raise ValueError("invalid boundary specification")

    def _z(self):
        return np.zeros(self.n_dofs)

    def vmult(self, src, T_lin=None, T_old=None, form=0):
        dst = self._z()
        T_lin = self._z() if T_lin is None else T_lin
        T_old = self._z() if T_old is None else T_old
        self.L.orc_vmult(self.h, _ptr(dst), _ptr(src), _ptr(T_lin), _ptr(T_old), form)
        return dst

    def inverse_diagonal(self, T_lin=None, T_old=None, form=0):
        d = self._z()
        T_lin = self._z() if T_lin is None else T_lin
        T_old = self._z() if T_old is None else T_old
        self.L.orc_inverse_diagonal(self.h, _ptr(d), _ptr(T_lin), _ptr(T_old), form)
        return d

    def create_rhs(self, T, T_old, heat_source=None, dst=None):
        dst = self._z() if dst is None else dst
        q = self._z() if heat_source is None else heat_source
        self.L.orc_create_rhs(self.h, _ptr(dst), _ptr(T), _ptr(T_old), _ptr(q))
        return dst

    def l2_norm(self, u):
        return float(self.L.orc_l2_norm(self.h, _ptr(u)))

    def cg(self, b, x=None, inv_diag=None, T_lin=None, T_old=None, rel_tol=1e-12, abs_tol=1e-20,
           max_it=10000, precond=1, cheb_degree=4, cheb_range=(0.0, 0.0)):
        x = self._z() if x is None else x
        T_lin = self._z() if T_lin is None else T_lin
        T_old = self._z() if T_old is None else T_old
        if inv_diag is None:
            inv_diag = self.inverse_diagonal(T_lin, T_old)
        p = SolverParams(max_it, rel_tol, abs_tol, precond, cheb_degree, cheb_range[0],
                         cheb_range[1])
        res = C.c_double(0.0)
        its = self.L.orc_cg(self.h, C.byref(p), _ptr(x), _ptr(b), _ptr(inv_diag), _ptr(T_lin),
                            _ptr(T_old), C.byref(res))
        return x, its, res.value

    def gmres(self, b, x=None, inv_diag=None, T_lin=None, T_old=None, rel_tol=1e-12,
              abs_tol=1e-20, max_it=10000, restart=28, precond=1):
        x = self._z() if x is None else x
        T_lin = self._z() if T_lin is None else T_lin
        T_old = self._z() if T_old is None else T_old
        if inv_diag is None:
            inv_diag = self.inverse_diagonal(T_lin, T_old)
        p = SolverParams(max_it, rel_tol, abs_tol, precond, 0, 0.0, 0.0)
        res = C.c_double(0.0)
        its = self.L.orc_gmres(self.h, C.byref(p), restart, _ptr(x), _ptr(b), _ptr(inv_diag),
                               _ptr(T_lin), _ptr(T_old), C.byref(res))
        return x, its, res.value

    def estimate_eigenvalues(self, inv_diag, T_lin=None, T_old=None, n_it=20):
        T_lin = self._z() if T_lin is None else T_lin
        T_old = self._z() if T_old is None else T_old
        lo, hi = C.c_double(), C.c_double()
        self.L.orc_estimate_eigenvalues(self.h, _ptr(inv_diag), _ptr(T_lin), _ptr(T_old), n_it,
                                        C.byref(lo), C.byref(hi))
        return lo.value, hi.value

    def chebyshev_apply(self, r, inv_diag, lam_min, lam_max, degree=4, T_lin=None, T_old=None):
        T_lin = self._z() if T_lin is None else T_lin
        T_old = self._z() if T_old is None else T_old
        p = SolverParams(0, 0.0, 0.0, 2, degree, lam_min, lam_max)
        x = self._z()
        self.L.orc_chebyshev_apply(self.h, C.byref(p), _ptr(x), _ptr(r), _ptr(inv_diag),
                                   _ptr(T_lin), _ptr(T_old))
        return x

    def linear_predictor(self, T_cur, T_old, dt, dt_old):
        pred = self._z()
        self.L.orc_linear_predictor(self.h, _ptr(T_cur), _ptr(T_old), _ptr(pred), dt, dt_old)
        return pred

    def time_step_newton(self, T_cur, T_old, dt, dt_old, heat_source=None, predictor=1,
                         rel_tol=1e-12, abs_tol=1e-20, max_it=10000, newton_max_it=10,
                         res_tol=1e-9, corr_tol=1e-10, solver="gmres"):
        q = self._z() if heat_source is None else heat_source
        lin = SolverParams(max_it, rel_tol, abs_tol, 1, 0, 0.0, 0.0)
        nl = NewtonParams(newton_max_it, res_tol, corr_tol)
        st = StepStats()
        rc = self.L.orc_time_step_newton(self.h, _ptr(T_cur), _ptr(T_old), _ptr(q), dt, dt_old,
                                         predictor, 1 if solver == "gmres" else 0, C.byref(lin), C.byref(nl), C.byref(st))
        return rc, st

    def laser_source(self, profile, power, position, radius=1.0, direction=(0.0, 0.0, -1.0),
                     gusarov=(0.0, 0.0, 0.0), planar=False):
        """Volumetric laser intensity at the support points (profile 0 uniform, 1 Gauss
        volumetric, 2 Gauss projection, 3 Gusarov with (reflectivity, extinction, layer));
        planar: the 2D profile in the x-z plane of a one-cell-thick mesh (y ignored)."""
        q = np.empty(self.n_dofs)
        c = np.ascontiguousarray(position, dtype=np.float64)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        self.L.orc_laser_source(self.h, _ptr(q), int(profile), float(power), _ptr(c), _ptr(d),
                                float(radius), *[float(v) for v in gusarov], int(bool(planar)))
        return q

    def gaussian_source(self, amp, center, radius):
        q = self._z()
        c = (C.c_double * 3)(*center)
        self.L.orc_gaussian_source(self.h, _ptr(q), amp, c, radius)
        return q


def set_threads(n: int):
    lib().orc_set_threads(int(n))
