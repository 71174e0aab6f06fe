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
