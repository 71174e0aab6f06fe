"""Heat operator on a box mesh with one level of refinement and hanging nodes (C ABI
mpdg_amr_*): the operator verbs of HeatDiffuseMultiPhaseOperator on the meshes MeltPoolDG's
refine_grid produces (source/utilities/amr.cpp:18-41), with the hanging-node constraints of
include/meltpooldg/utilities/constraints.hpp:111-132 applied inside the cell kernel."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .heat import ExcInvalidArgument, check


class AmrHeatOperator:
    """refine: coarse cell indices (ix, iy, iz) to split once, a bool array [mz][my][mx], or an
    integer array [mz][my][mx] of refinement levels (2:1 balanced; one level on a device).
    device=None builds the host description only (DoFs, support points, cell data)."""

    def __init__(self, mesh: L.MeshDesc, refine=(), device: int | None = 0):
        self._L = L.load()
        m = tuple(mesh.cells)
        ref = np.zeros((m[2], m[1], m[0]), dtype=np.uint8)
        if isinstance(refine, np.ndarray) and refine.dtype.kind in "biu":
            ref[...] = refine.astype(np.uint8)
        else:
            for ix, iy, iz in refine:
                ref[iz, iy, ix] = 1
        self._refine = np.ascontiguousarray(ref)
        self.mesh = mesh
        self.device = None if device is None else torch.device("cuda", device)
        h = C.c_void_p()
        check(self._L.mpdg_amr_create(C.byref(mesh), self._refine.ctypes.data_as(C.c_void_p),
                                      -1 if device is None else int(device), C.byref(h)))
        self.h = h
        self.n_dofs = int(self._L.mpdg_amr_n_dofs(h))
        self.n_cells = int(self._L.mpdg_amr_n_cells(h))
        self.n = mesh.degree + 1

    def __del__(self):
        try:
            if self.h:
                self._L.mpdg_amr_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def support_points(self) -> np.ndarray:
        x = np.empty((self.n_dofs, 3))
        check(self._L.mpdg_amr_support_points(self.h, x.ctypes.data_as(C.c_void_p)))
        return x

    def constraint_mask(self) -> np.ndarray:
        mk = np.empty(self.n_dofs, dtype=np.uint8)
        check(self._L.mpdg_amr_constraint_mask(self.h, mk.ctypes.data_as(C.c_void_p)))
        return mk

    def cell_data(self):
        dofs = np.empty((self.n_cells, self.n ** 3), dtype=np.int64)
        codes = np.empty(self.n_cells, dtype=np.uint16)
        check(self._L.mpdg_amr_cell_data(self.h, dofs.ctypes.data_as(C.c_void_p),
                                         codes.ctypes.data_as(C.c_void_p)))
        return dofs, codes

    def set_material(self, m: L.Material, dt: float):
        check(self._L.mpdg_amr_set_material(self.h, C.byref(m), float(dt)))

    def vmult(self, dst: torch.Tensor, src: torch.Tensor, T_lin: torch.Tensor | None = None):
        for t in (dst, src) + (() if T_lin is None else (T_lin,)):
            if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous() or \
                    t.numel() != self.n_dofs:
                raise ExcInvalidArgument("expected contiguous CUDA float64 vectors of n_dofs")
        torch.cuda.current_stream().synchronize()  # the kernel runs on the legacy stream
        check(self._L.mpdg_amr_vmult(self.h, dst.data_ptr(), src.data_ptr(),
                                     None if T_lin is None else T_lin.data_ptr()))

    def _vec(self, *ts):
        for t in ts:
            if t is None:
                continue
            if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous() or \
                    t.numel() != self.n_dofs:
                raise ExcInvalidArgument("expected contiguous CUDA float64 vectors of n_dofs")
        torch.cuda.current_stream().synchronize()  # the kernels run on the legacy stream
        return [None if t is None else t.data_ptr() for t in ts]

    def inverse_diagonal(self, inv_diag: torch.Tensor, T_lin: torch.Tensor | None = None):
        """compute_inverse_diagonal_from_matrixfree on the refined mesh."""
        check(self._L.mpdg_amr_inverse_diagonal(self.h, *self._vec(inv_diag, T_lin)))
        return inv_diag

    def create_rhs(self, dst, T, T_old, heat_source=None):
        """dst += -R(T) (T the linearisation point, T_old the previous step)."""
        check(self._L.mpdg_amr_create_rhs(self.h, *self._vec(dst, T, T_old, heat_source)))
        return dst

    def linear_solve(self, x, b, T_lin=None, rel_tolerance=1e-12, abs_tolerance=1e-20,
                     max_iterations=10000) -> int:
        """Jacobi-CG from x = 0; returns the iteration count."""
        its = C.c_int()
        check(self._L.mpdg_amr_linear_solve(self.h, *self._vec(x, b, T_lin), float(rel_tolerance),
                                            float(abs_tolerance), int(max_iterations),
                                            C.byref(its)))
        return int(its.value)

    def time_step(self, T_cur, T_old, dt, dt_old, heat_source=None, params=None) -> L.StepStats:
        """HeatDiffuseOperation::solve on the refined mesh (T_cur, T_old updated in place)."""
        from .heat import step_params
        prm = params if params is not None else step_params()
        st = L.StepStats()
        a, b, q = self._vec(T_cur, T_old, heat_source)
        check(self._L.mpdg_amr_time_step(self.h, float(dt), float(dt_old), a, b, q,
                                         C.byref(prm), C.byref(st)))
        return st
