"""Python mirror of MeltPoolDG's heat-operator interface over the C ABI.

Names, argument meaning and error behaviour follow the reference:
  HeatDiffuseOperator   HeatDiffuseMultiPhaseOperator / OperatorMatrixFree verbs
                        (include/meltpooldg/core/operator_base.hpp:188-282)
  JacobiPreconditioner  include/meltpooldg/linear_algebra/preconditioner_jacobi.hpp
  LinearSolver.solve    include/meltpooldg/linear_algebra/linear_solver.hpp:22-134
  HeatDiffuseOperation  source/heat/heat_diffuse_operation.cpp (init_time_advance + solve)
Vectors are torch CUDA tensors (float64, or float32 for the FP32 operator) of
length n_dofs; all work runs on the CUDA library (libmpdg_heat.so), there is no
CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import torch

from . import _lib as L


# ---------------------------------------------------------------------------
# exceptions (deal.II / MeltPoolDG exception names)
# ---------------------------------------------------------------------------
class MpdgError(RuntimeError):
    code = -1


class ExcInvalidArgument(MpdgError, ValueError):
    code = L.ERR_INVALID_ARGUMENT


class ExcOutOfMemory(MpdgError, MemoryError):
    code = L.ERR_OUT_OF_MEMORY


class ExcNoConvergence(MpdgError):
    """dealii::SolverControl::NoConvergence."""
    code = L.ERR_NOT_CONVERGED


class ExcNaN(ExcNoConvergence):
    code = L.ERR_NAN


class ExcBreakdown(ExcNoConvergence):
    code = L.ERR_BREAKDOWN


class ExcCuda(MpdgError):
    code = L.ERR_CUDA


class ExcZeroTimeIncrement(MpdgError):
    """AssertThrowZeroTimeIncrement (include/meltpooldg/core/exceptions.hpp:6)."""
    code = L.ERR_ZERO_TIME_INCREMENT


class ExcHeatTransferNoConvergence(MpdgError):
    """ExcNewtonDidNotConverge -> ExcHeatTransferNoConvergence (exceptions.hpp:25-26)."""
    code = L.ERR_NEWTON_NOT_CONVERGED


class ExcNotImplemented(MpdgError, NotImplementedError):
    code = L.ERR_NOT_SUPPORTED


_EXC = {c.code: c for c in (ExcInvalidArgument, ExcOutOfMemory, ExcNoConvergence, ExcNaN,
                             ExcBreakdown, ExcCuda, ExcZeroTimeIncrement,
                             ExcHeatTransferNoConvergence, ExcNotImplemented)}


def check(rc: int):
    if rc != L.OK:
        raise _EXC.get(rc, MpdgError)(f"[{rc}] {L.last_error()}")


# ---------------------------------------------------------------------------
# descriptions
# ---------------------------------------------------------------------------
FACES = {"x-": 0, "x+": 1, "y-": 2, "y+": 3, "z-": 4, "z+": 5}


def box_mesh(degree, cells, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), perturb=0.0, seed=1,
             dirichlet=("x-", "x+", "y-", "y+", "z-", "z+"), dirichlet_values=None) -> L.MeshDesc:
    """Structured FE_Q(degree) box mesh; `dirichlet` lists constrained faces."""
    d = L.MeshDesc()
    d.degree = int(degree)
    for i in range(3):
        d.cells[i] = int(cells[i])
        d.lo[i] = float(lo[i])
        d.hi[i] = float(hi[i])
    d.perturb = float(perturb)
    d.seed = int(seed)
    mask = 0
    for f in dirichlet:
        mask |= 1 << (FACES[f] if isinstance(f, str) else int(f))
    d.dirichlet_mask = mask
    vals = dirichlet_values or {}
    for f, v in (vals.items() if isinstance(vals, dict) else enumerate(vals)):
        d.dirichlet_value[FACES[f] if isinstance(f, str) else int(f)] = float(v)
    return d


def material(law=L.LAW_CONSTANT, rho=1.0, cp=1.0, k=1.0, k1=0.0, rho_s=None, cp_s=None, k_s=None,
             T_solidus=0.0, T_liquidus=1.0, sharp=False, volume_specific=False, rho_g=None,
             cp_g=None, k_g=None, sharp_gas_liquid=False) -> L.Material:
    """Material parameters: liquid (rho, cp, k), solid (*_s) and gas (*_g) phases, each
    defaulting to the liquid values; sharp selects the sharp liquid-solid transition,
    sharp_gas_liquid the sharp gas-liquid one."""
    m = L.Material()
    m.law = int(law)
    m.sharp = int(sharp)
    m.volume_specific = int(volume_specific)
    m.rho_l, m.cp_l, m.k_l = float(rho), float(cp), float(k)
    m.rho_s = float(rho if rho_s is None else rho_s)
    m.cp_s = float(cp if cp_s is None else cp_s)
    m.k_s = float(k if k_s is None else k_s)
    m.T_solidus, m.T_liquidus, m.k1 = float(T_solidus), float(T_liquidus), float(k1)
    m.sharp_gas_liquid = int(sharp_gas_liquid)
    m.rho_g = float(rho if rho_g is None else rho_g)
    m.cp_g = float(cp if cp_g is None else cp_g)
    m.k_g = float(k if k_g is None else k_g)
    return m


def material_eval(m: L.Material, T: float, H: float = 1.0, latent_heat: float = 0.0,
                  profile: int = L.APPARENT_QLQ):
    """(rho*cp, k, d(rho*cp)/dT, dk/dT) of the law at temperature T and heaviside H, evaluated
    on the host by the code the cell kernels run (mpdg_material_eval; no GPU needed)."""
    out = (C.c_double * 4)()
    check(L.load().mpdg_material_eval(C.byref(m), float(latent_heat), int(profile), float(T),
                                      float(H), out))
    return tuple(out)


@dataclass
class LinearSolverData:
    """LinearSolverData (linear_solver_data.hpp:40-47) plus the Chebyshev and multigrid options."""
    solver_type: int = L.SOLVER_CG
    preconditioner_type: int = L.PRECOND_JACOBI
    max_iterations: int = 10000
    rel_tolerance: float = 1e-12
    abs_tolerance: float = 1e-20
    gmres_restart: int = 28
    cheb_degree: int = 4
    cheb_eig_iterations: int = 12
    cheb_max_factor: float = 1.2
    cheb_min_fraction: float = 0.0
    tol_reference_norm: float = 0.0
    cheb_picard: bool = False
    cheb_eig_reuse: bool = False
    mg_smoothing_degree: int = 2
    mg_coarse_degree: int = 8
    mg_smoothing_range: float = 8.0
    mg_min_cells: int = 4
    mg_fine_pre_steps: int = -1
    mg_fine_post_steps: int = -1

    def to_c(self) -> L.SolverParams:
        return L.SolverParams(self.solver_type, self.preconditioner_type, self.max_iterations,
                              self.rel_tolerance, self.abs_tolerance, self.gmres_restart,
                              self.cheb_degree, self.cheb_eig_iterations, self.cheb_max_factor,
                              self.cheb_min_fraction, self.tol_reference_norm,
                              int(self.cheb_picard), int(self.cheb_eig_reuse),
                              self.mg_smoothing_degree, self.mg_coarse_degree,
                              self.mg_smoothing_range, self.mg_min_cells,
                              self.mg_fine_pre_steps, self.mg_fine_post_steps)


@dataclass
class NonlinearSolverData:
    """NonlinearSolverData (nonlinear_solver_data.hpp:13-19)."""
    max_nonlinear_iterations: int = 10
    residual_tolerance: float = 1e-9
    field_correction_tolerance: float = 1e-10


def _ptr(t: torch.Tensor | None, dtype=torch.float64):
    if t is None:
        return None
    if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
        raise ExcInvalidArgument(f"expected a contiguous CUDA {dtype} tensor, got "
                                 f"{t.dtype} on {t.device}")
    return t.data_ptr()


def _host_ptr(a, n=None, dtype=None):
    """Data pointer of a contiguous host array (numpy or CPU torch) of n float64 values."""
    if a is None:
        return None
    import numpy as np
    if isinstance(a, torch.Tensor):
        if a.is_cuda or not a.is_contiguous() or a.dtype != (dtype or torch.float64):
            raise ExcInvalidArgument("expected a contiguous host tensor")
        size, ptr = a.numel(), a.data_ptr()
    else:
        want = np.int64 if dtype is torch.int64 else np.float64
        if not isinstance(a, np.ndarray) or a.dtype != want or not a.flags.c_contiguous:
            raise ExcInvalidArgument(f"expected a contiguous {want.__name__} numpy array")
        size, ptr = a.size, a.ctypes.data
    if n is not None and size != n:
        raise ExcInvalidArgument(f"expected {n} values, got {size}")
    return C.c_void_p(ptr)


# ---------------------------------------------------------------------------
# operator
# ---------------------------------------------------------------------------
class HeatDiffuseOperator:
    """Matrix-free heat tangent operator on one GPU (OperatorMatrixFree verbs)."""

    def __init__(self, mesh: L.MeshDesc, device: int = 0, slab=None):
        """slab=(z_begin, z_end): this rank's z-slab of cells of the global mesh `mesh`
        (mpdg_heat_create_slab); the shared end planes are summed by the caller."""
        self._L = L.load()
        # a private copy: set_dirichlet_values changes this operator's values only, not the
        # caller's descriptor (which may also describe an oracle, a slab or another operator)
        self.mesh = L.MeshDesc.from_buffer_copy(mesh)
        mesh = self.mesh
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        if slab is None:
            check(self._L.mpdg_heat_create(C.byref(mesh), device, C.byref(h)))
        else:
            check(self._L.mpdg_heat_create_slab(C.byref(mesh), int(slab[0]), int(slab[1]),
                                                device, C.byref(h)))
        self.h = h
        n = C.c_int64()
        check(self._L.mpdg_heat_n_dofs(h, C.byref(n)))
        self.n_dofs = int(n.value)
        check(self._L.mpdg_heat_n_cells(h, C.byref(n)))
        self.n_cells = int(n.value)
        dims = (C.c_int * 3)()
        check(self._L.mpdg_heat_dof_dims(h, dims))
        self.dims = tuple(dims)
        self.degree = mesh.degree
        self._refs = ()
        self.sync_stream()

    def sync_stream(self):
        """Enqueue subsequent work on torch's current stream of this device."""
        with torch.cuda.device(self.device):
            s = torch.cuda.current_stream().cuda_stream
        check(self._L.mpdg_heat_set_stream(self.h, C.c_void_p(s)))

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self._L.mpdg_heat_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def new_vector(self, dtype=torch.float64):
        return torch.zeros(self.n_dofs, dtype=dtype, device=self.device)

    def device_bytes(self) -> int:
        n = C.c_int64()
        check(self._L.mpdg_heat_device_bytes(self.h, C.byref(n)))
        return int(n.value)

    # coefficients ---------------------------------------------------------
    def set_material(self, m: L.Material):
        check(self._L.mpdg_heat_set_material(self.h, C.byref(m)))

    def set_latent_heat(self, latent_heat: float, profile: int = L.APPARENT_QLQ):
        """Latent heat of fusion as an apparent heat capacity in the mushy zone
        (MaterialData::latent_heat_of_fusion, apparent_capacity_type); 0 switches it off."""
        check(self._L.mpdg_heat_set_latent_heat(self.h, float(latent_heat), int(profile)))

    def set_dirichlet_values(self, values):
        """Dirichlet values per face for the following steps (a dict {"x-": v, ...} over the
        Dirichlet faces, or six values in the order x-, x+, y-, y+, z-, z+)."""
        v = (C.c_double * 6)()
        if isinstance(values, dict):
            cur = list(self.mesh.dirichlet_value)
            for f, val in values.items():
                cur[FACES[f]] = float(val)
            values = cur
        for i, val in enumerate(values):
            v[i] = float(val)
        check(self._L.mpdg_heat_set_dirichlet_values(self.h, v))
        for i in range(6):
            self.mesh.dirichlet_value[i] = v[i]

    def set_fields(self, heaviside=None, velocity=None):
        """Level-set heaviside (n_dofs) and velocity ((3, n_dofs), component-major) fields
        of the two-phase operator, torch CUDA float64 tensors on this operator's DoFs; None
        removes one. Call again after changing a field's contents."""
        if velocity is not None:
            assert velocity.is_contiguous() and velocity.numel() == 3 * self.n_dofs
        self._fields = (heaviside, velocity)
        check(self._L.mpdg_heat_set_fields(self.h, _ptr(heaviside), _ptr(velocity)))

    def set_boundary(self, face, convection=None, radiation=None, neumann=None):
        """Robin / Neumann terms on a box face: convection=(h, T_inf),
        radiation=(emissivity, T_inf), neumann=q_n; no argument clears the face."""
        f = FACES[face] if isinstance(face, str) else int(face)
        t = (1 if convection else 0) | (2 if radiation else 0) | (4 if neumann is not None else 0)
        hc, tc = convection or (0.0, 0.0)
        e, tr = radiation or (0.0, 0.0)
        check(self._L.mpdg_heat_set_boundary(self.h, f, t, float(hc), float(tc), float(e),
                                              float(tr), 0.0 if neumann is None else float(neumann)))

    def reset_time_increment(self, dt: float):
        check(self._L.mpdg_heat_reset_time_increment(self.h, float(dt)))

    def set_linearization(self, temperature, temperature_old=None):
        self._refs = (temperature, temperature_old)
        check(self._L.mpdg_heat_set_linearization(self.h, _ptr(temperature),
                                                   _ptr(temperature_old)))

    # verbs ------------------------------------------------------------------
    def vmult(self, dst, src):
        if src.dtype == torch.float32:
            check(self._L.mpdg_heat_vmult_f32(self.h, _ptr(dst, torch.float32),
                                               _ptr(src, torch.float32)))
        else:
            check(self._L.mpdg_heat_vmult(self.h, _ptr(dst), _ptr(src)))
        return dst

    def vmult_picard_f32(self, dst, src):
        """FP32 Picard operator of the mixed-precision preconditioner: the tangent of the
        linear-k law with k(T_lin) frozen at the quadrature points (no dk/dT term)."""
        check(self._L.mpdg_heat_vmult_f32_picard(self.h, _ptr(dst, torch.float32),
                                                  _ptr(src, torch.float32)))
        return dst

    def cell_rows_size(self) -> int:
        """Floats of an FP32 vector in the cell-row layout (FE_Q(3)): 4 slots per cell of each
        x-row of the nodal grid, the node shared by x-neighbouring cells stored in both."""
        n = C.c_int64(0)
        check(self._L.mpdg_heat_cell_rows_size(self.h, C.byref(n)))
        return int(n.value)

    def to_cell_rows_f32(self, rows, lex):
        """rows = the cell-row copy of the lexicographic FP32 vector lex."""
        check(self._L.mpdg_heat_to_cell_rows_f32(self.h, _ptr(rows, torch.float32),
                                                  _ptr(lex, torch.float32)))
        return rows

    def vmult_picard_f32_rows(self, dst, src_rows):
        """The FP32 Picard operator applied to an operand in the cell-row layout (the kernel of
        the multigrid's fine level); dst is lexicographic."""
        check(self._L.mpdg_heat_vmult_f32_picard_rows(self.h, _ptr(dst, torch.float32),
                                                       _ptr(src_rows, torch.float32)))
        return dst

    @property
    def picard_cell_rows(self) -> bool:
        """True when the last mixed-precision solve kept the fine level's Chebyshev iterate in
        the cell-row layout (the Picard operator's vector gather)."""
        return bool(self._L.mpdg_heat_picard_cell_rows(self.h))

    def set_picard_tensor_cores(self, on: bool):
        """Apply the FP32 Picard operator on the tensor cores (TF32 operands) where the kernel
        exists (uniform box, FE_Q(3)); off (the default) keeps the CUDA-core kernel."""
        check(self._L.mpdg_heat_set_picard_tensor_cores(self.h, int(bool(on))))

    @property
    def picard_tensor_cores(self) -> bool:
        return bool(self._L.mpdg_heat_picard_tensor_cores(self.h))

    def inverse_diagonal_picard_f32(self, inv_diag):
        """Inverse diagonal of the FP32 Picard operator (the multigrid smoothers' scaling)."""
        check(self._L.mpdg_heat_inverse_diagonal_f32_picard(self.h, _ptr(inv_diag, torch.float32)))
        return inv_diag

    def compute_inverse_diagonal_from_matrixfree(self, diag):
        check(self._L.mpdg_heat_compute_inverse_diagonal(self.h, _ptr(diag)))
        return diag

    def compute_diagonal(self, diag):
        """diag(J), not inverted (constrained rows 0)."""
        check(self._L.mpdg_heat_compute_diagonal(self.h, _ptr(diag)))
        return diag

    def create_rhs(self, dst, src, heat_source=None):
        check(self._L.mpdg_heat_create_rhs(self.h, _ptr(dst), _ptr(src), _ptr(heat_source)))
        return dst

    def distribute_constraints(self, u):
        check(self._L.mpdg_heat_distribute_constraints(self.h, _ptr(u)))
        return u

    # stages of a Jacobi-CG iteration split across ranks (the caller all-reduces `partial`
    # between stages; alpha, beta and the partial sums are device tensors) ------------------
    def dcg_start(self, n_owned, b, Ax, inv_diag, r, z, p, partial):
        check(self._L.mpdg_heat_dcg_start(self.h, int(n_owned), _ptr(b), _ptr(Ax), _ptr(inv_diag),
                                          _ptr(r), _ptr(z), _ptr(p), _ptr(partial)))

    def dcg_dot(self, n_owned, a, b, partial):
        check(self._L.mpdg_heat_dcg_dot(self.h, int(n_owned), _ptr(a), _ptr(b), _ptr(partial)))

    def dcg_update(self, n_owned, x, r, z, p, Ap, inv_diag, alpha, partial):
        check(self._L.mpdg_heat_dcg_update(self.h, int(n_owned), _ptr(x), _ptr(r), _ptr(z),
                                           _ptr(p), _ptr(Ap), _ptr(inv_diag), _ptr(alpha),
                                           _ptr(partial)))

    def dcg_direction(self, p, z, beta):
        check(self._L.mpdg_heat_dcg_direction(self.h, _ptr(p), _ptr(z), _ptr(beta)))

    def invert_diagonal(self, d):
        """d <- |d| > 1e-10 ? 1/d : 1 (compute_inverse_diagonal_from_matrixfree's rule)."""
        check(self._L.mpdg_heat_invert_diagonal(self.h, _ptr(d)))
        return d

    # verbs on host vectors (OperatorMatrixFree's VectorType lives in host memory) --------
    def set_dof_permutation(self, lex_of_dof):
        """The caller's DoF numbering: lex_of_dof[i] is the lexicographic index of the
        caller's DoF i (int64 host array); None restores the identity."""
        self._perm = lex_of_dof
        check(self._L.mpdg_heat_set_dof_permutation(
            self.h, _host_ptr(lex_of_dof, self.n_dofs, torch.int64)))

    def set_linearization_host(self, temperature, temperature_old=None):
        check(self._L.mpdg_heat_set_linearization_host(
            self.h, _host_ptr(temperature, self.n_dofs), _host_ptr(temperature_old, self.n_dofs)))

    def vmult_host(self, dst, src):
        check(self._L.mpdg_heat_vmult_host(self.h, _host_ptr(dst, self.n_dofs),
                                           _host_ptr(src, self.n_dofs)))
        return dst

    def compute_inverse_diagonal_host(self, diag):
        check(self._L.mpdg_heat_compute_inverse_diagonal_host(self.h, _host_ptr(diag, self.n_dofs)))
        return diag

    def create_rhs_host(self, dst, src, heat_source=None):
        check(self._L.mpdg_heat_create_rhs_host(self.h, _host_ptr(dst, self.n_dofs),
                                                _host_ptr(src, self.n_dofs),
                                                _host_ptr(heat_source, self.n_dofs)))
        return dst

    def l2_norm(self, u) -> float:
        v = C.c_double()
        check(self._L.mpdg_heat_l2_norm(self.h, _ptr(u), C.byref(v)))
        return float(v.value)

    def set_timing(self, enable: bool):
        check(self._L.mpdg_heat_set_timing(self.h, int(bool(enable))))

    def counters(self, reset: bool = False) -> dict:
        c = L.Counters()
        check(self._L.mpdg_heat_get_counters(self.h, C.byref(c), int(bool(reset))))
        return {k: getattr(c, k) for k, _ in L.Counters._fields_}

    def support_points(self):
        x = torch.empty((self.n_dofs, 3), dtype=torch.float64, device=self.device)
        check(self._L.mpdg_heat_support_points(self.h, x.data_ptr()))
        return x

    def laser_source(self, q, profile, power, position, radius=1.0, direction=(0.0, 0.0, -1.0),
                     gusarov=(0.0, 0.0, 0.0), planar=False):
        """LaserHeatSourceVolumetric::compute_volumetric_heat_source: q = I(x) at the
        support points for profile L.LASER_UNIFORM / _GAUSS_VOLUMETRIC / _GAUSS_PROJECTION /
        _GUSAROV (gusarov = (reflectivity, extinction coefficient, layer thickness));
        planar: the 2D profile in the x-z plane of a mesh one cell thick in y."""
        las = L.Laser(int(profile), float(power), (C.c_double * 3)(*map(float, position)),
                      (C.c_double * 3)(*map(float, direction)), float(radius),
                      *[float(v) for v in gusarov], int(bool(planar)))
        check(self._L.mpdg_heat_laser_source(self.h, _ptr(q), C.byref(las)))
        return q

    def set_laser(self, profile=None, power=0.0, position=(0.0, 0.0, 0.0), radius=1.0,
                  direction=(0.0, 0.0, -1.0), gusarov=(0.0, 0.0, 0.0), planar=False):
        """The laser as the residual's source, evaluated inside the create_rhs kernels wherever
        the heat source is None (profile None switches it off)."""
        if profile is None:
            check(self._L.mpdg_heat_set_laser(self.h, None))
            return
        las = L.Laser(int(profile), float(power), (C.c_double * 3)(*map(float, position)),
                      (C.c_double * 3)(*map(float, direction)), float(radius),
                      *[float(v) for v in gusarov], int(bool(planar)))
        check(self._L.mpdg_heat_set_laser(self.h, C.byref(las)))

    def gaussian_source(self, q, amplitude, center, radius):
        c = (C.c_double * 3)(*[float(v) for v in center])
        check(self._L.mpdg_heat_gaussian_source(self.h, _ptr(q), float(amplitude), c,
                                                 float(radius)))
        return q


class JacobiPreconditioner:
    """JacobiPreconditioner: update() stores inv diag(J) in the handle; vmult scales."""

    def __init__(self, op: HeatDiffuseOperator):
        self.op = op

    def update(self, *_):
        check(self.op._L.mpdg_heat_preconditioner_update(self.op.h))

    def vmult(self, dst, src):
        check(self.op._L.mpdg_heat_preconditioner_vmult(self.op.h, _ptr(dst), _ptr(src)))
        return dst

    def reinit(self):
        pass


class LinearSolver:
    last_stats: L.SolveStats | None = None

    @staticmethod
    def solve(op: HeatDiffuseOperator, solution, rhs, data: LinearSolverData = None,
              preconditioner=None) -> int:
        """Solve J x = b from the guess in `solution`; returns the iteration count and
        raises ExcNoConvergence like dealii::SolverControl::NoConvergence."""
        data = data or LinearSolverData()
        if preconditioner is None and data.preconditioner_type != L.PRECOND_IDENTITY:
            data = LinearSolverData(**{**data.__dict__, "preconditioner_type": L.PRECOND_IDENTITY})
        prm = data.to_c()
        st = L.SolveStats()
        rc = op._L.mpdg_heat_linear_solve(op.h, C.byref(prm), _ptr(solution), _ptr(rhs),
                                          C.byref(st))
        LinearSolver.last_stats = st
        check(rc)
        return int(st.iterations)


def step_params(linear: LinearSolverData = None, nonlinear: NonlinearSolverData = None,
                predictor=L.PREDICTOR_LINEAR, single_linearization=False) -> L.StepParams:
    linear = linear or LinearSolverData()
    nonlinear = nonlinear or NonlinearSolverData()
    p = L.StepParams()
    p.newton_max_iterations = nonlinear.max_nonlinear_iterations
    p.newton_residual_tolerance = nonlinear.residual_tolerance
    p.newton_correction_tolerance = nonlinear.field_correction_tolerance
    p.predictor = int(predictor)
    p.single_linearization = int(bool(single_linearization))
    p.linear = linear.to_c()
    return p


class HeatDiffuseOperation:
    """HeatDiffuseOperation: owns the solution history on the device and advances it.

    solve(dt) = init_time_advance (predictor, history commit, constraints) +
    preconditioner update + Newton-Raphson (heat_diffuse_operation.cpp:213-289).
    """

    def __init__(self, op: HeatDiffuseOperator, linear: LinearSolverData = None,
                 nonlinear: NonlinearSolverData = None, predictor=L.PREDICTOR_LINEAR,
                 single_linearization=False):
        self.op = op
        self.params = step_params(linear, nonlinear, predictor, single_linearization)
        self.T = op.new_vector()
        self.T_old = op.new_vector()
        self.heat_source = None
        self.dt_old = 0.0
        self.last_stats = None

    def set_initial_condition(self, T0):
        self.T.copy_(T0)
        self.op.distribute_constraints(self.T)

    def set_guess(self, guess):
        check(self.op._L.mpdg_heat_set_guess(self.op.h, _ptr(guess)))
        self._guess = guess

    def set_direction(self, direction):
        """Increment direction for PREDICTOR_LINEAR_DIRECTION (zero at Dirichlet DoFs)."""
        check(self.op._L.mpdg_heat_set_direction(self.op.h, _ptr(direction)))
        self._direction = direction

    # host-buffer steps with the history resident on the device --------------------------
    @staticmethod
    def _host_ptr(t):
        if t is None:
            return None
        if t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
            raise ExcInvalidArgument("expected a contiguous host float64 tensor")
        return C.c_void_p(t.data_ptr())

    def load_history_host(self, T, T_old):
        """Copy host T and T_old into the operator's device-resident history."""
        check(self.op._L.mpdg_heat_load_history(self.op.h, self._host_ptr(T),
                                                self._host_ptr(T_old)))

    def store_history_host(self, T=None, T_old=None):
        check(self.op._L.mpdg_heat_store_history(self.op.h, self._host_ptr(T),
                                                 self._host_ptr(T_old)))

    def solve_resident(self, dt: float, heat_source_host=None, T_out_host=None):
        """One step on the resident history: uploads the host source, returns the new T
        into T_out_host (pinned host tensors overlap the copies with the step)."""
        st = L.StepStats()
        rc = self.op._L.mpdg_heat_time_step_resident(
            self.op.h, C.byref(self.params), float(dt), float(self.dt_old),
            self._host_ptr(heat_source_host), self._host_ptr(T_out_host), C.byref(st))
        self.last_stats = st
        check(rc)
        self.dt_old = float(dt)
        return st

    def solve(self, dt: float):
        st = L.StepStats()
        rc = self.op._L.mpdg_heat_time_step(self.op.h, C.byref(self.params), float(dt),
                                            float(self.dt_old), _ptr(self.T), _ptr(self.T_old),
                                            _ptr(self.heat_source), C.byref(st))
        self.last_stats = st
        check(rc)
        self.dt_old = float(dt)
        return st
