"""Time the hanging-node operator (mpdg_amr_*) on a refined box mesh.

    python bench_amr.py [--degree 3] [--cells 48] [--reps 10]

The mesh: the unit cube with `cells`^3 coarse cells, the coarse cells of the central half of the
box in every direction refined once (an eighth of the volume at twice the resolution, hanging
faces, edges and corners around it), Dirichlet on all faces, k(T) = 1 + 0.5 T. Prints one JSON
line: the CUDA-event time per operator application (FP64 linear-k tangent), per inverse diagonal,
per create_rhs, and per implicit step (Jacobi-CG to 1e-8), with the DoF count, the structured
operator's time on the unrefined mesh of the same coarse cells for comparison, and DoFs per second.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from meltpooldg_b200.amr import AmrHeatOperator


def timed(fn, reps):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--degree", type=int, default=3)
    ap.add_argument("--cells", type=int, default=48)
    ap.add_argument("--reps", type=int, default=10)
    a = ap.parse_args()
    m = a.cells
    ref = np.zeros((m, m, m), dtype=np.uint8)
    q0, q1 = m // 4, m - m // 4
    ref[q0:q1, q0:q1, q0:q1] = 1
    mesh = H.box_mesh(a.degree, (m, m, m))
    op = AmrHeatOperator(mesh, ref, device=0)
    dt = 5e-4
    op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5), dt)
    N = op.n_dofs
    g = torch.Generator(device="cuda").manual_seed(0)
    T = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
    x = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
    y = torch.empty_like(x)
    ms_vmult = timed(lambda: op.vmult(y, x, T), a.reps)
    ms_diag = timed(lambda: op.inverse_diagonal(y, T), max(2, a.reps // 5))
    q = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
    ms_rhs = timed(lambda: op.create_rhs(y, T, T, q), a.reps)
    # implicit steps from T = 0 with a source: Jacobi-CG increment solves to 1e-8
    prm = H.step_params()
    prm.linear.rel_tolerance = 1e-8
    prm.linear.abs_tolerance = 0.0
    Tc = torch.zeros(N, dtype=torch.float64, device="cuda")
    To = torch.zeros_like(Tc)
    stats = []

    def step():
        stats.append(op.time_step(Tc, To, dt, dt, 100.0 * q, prm))
    ms_step = timed(step, 3)
    its = [s.linear_iterations for s in stats]
    # the structured operator on the unrefined mesh of the same coarse cells
    sop = H.HeatDiffuseOperator(mesh)
    sop.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
    sop.reset_time_increment(dt)
    Ns = sop.n_dofs
    Ts = torch.rand(Ns, dtype=torch.float64, device="cuda", generator=g)
    xs = torch.rand(Ns, dtype=torch.float64, device="cuda", generator=g)
    ys = torch.empty_like(xs)
    sop.set_linearization(Ts, Ts)
    ms_struct = timed(lambda: sop.vmult(ys, xs), a.reps)
    print(json.dumps({"degree": a.degree, "coarse_cells": m, "active_cells": op.n_cells,
                      "n_dofs": N, "refined_fraction_of_volume": float(ref.mean()),
                      "vmult_ms": ms_vmult, "vmult_gdofs": N / ms_vmult / 1e6,
                      "inverse_diagonal_ms": ms_diag, "create_rhs_ms": ms_rhs,
                      "step_ms": ms_step, "step_cg_iterations": its[-3:],
                      "structured_unrefined": {"n_dofs": Ns, "vmult_ms": ms_struct,
                                               "vmult_gdofs": Ns / ms_struct / 1e6}}), flush=True)


if __name__ == "__main__":
    main()
