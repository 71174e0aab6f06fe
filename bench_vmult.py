"""Time (and give ncu a target for) the operator application on one mesh.

  python bench_vmult.py --degree 3 --cells 96 --law 1 --reps 3
prints one JSON line per precision with the CUDA-event time per application,
DoFs/s and algorithmic GB/s (src + dst + linearisation point [+ per-q geometry]).
With --solve it instead runs a few outer iterations of FP64 CG with the FP32
Chebyshev preconditioner on the Picard operator, so that kernel can be captured.
With --picard it times the FP32 Picard operator of the multigrid fine level (conductivity
frozen at the quadrature points; src + dst + the conductivity per point in the traffic), on
the tensor cores where that kernel exists and on the CUDA cores, one line each.
With --transport the operator is the two-phase one (gas-liquid law on a heaviside
field plus the convective term of a velocity field), whose per-point coefficients
(5 per quadrature point) replace the linearisation point in the traffic;
--transport --law 4 uses the three-phase law (liquid-solid at T_lin mixed with the
gas): where the register-resident kernel exists (p <= 3 FP64, p <= 4 FP32) its 8
tangent coefficients per point are built once per linearisation (reported as
setup_ms, the first application minus a steady one) and the application reads src,
dst and the coefficients; elsewhere the line-per-thread kernel reads src, dst, T_lin,
T_old and 5 field values per point.
"""
from __future__ import annotations

import argparse
import json

import torch

from meltpooldg_b200 import heat as H


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--degree", type=int, default=3)
    ap.add_argument("--cells", type=int, default=96)
    ap.add_argument("--perturb", type=float, default=0.0)
    ap.add_argument("--law", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--dtype", default="both", choices=["f64", "f32", "both"])
    ap.add_argument("--solve", action="store_true")
    ap.add_argument("--transport", action="store_true")
    ap.add_argument("--picard", action="store_true")
    a = ap.parse_args()
    op = H.HeatDiffuseOperator(H.box_mesh(a.degree, (a.cells,) * 3, perturb=a.perturb))
    if a.transport:
        a.law = 4 if a.law == 4 else 3
        op.set_material(H.material(law=a.law, rho=2.0, cp=3.0, k=5.0, rho_s=2.2, cp_s=2.5, k_s=4.0,
                                   T_solidus=0.3, T_liquidus=0.7, rho_g=0.5, cp_g=1.5, k_g=0.3))
    else:
        op.set_material(H.material(law=a.law, k=1.0, k1=0.5))
    op.reset_time_increment(5e-4)
    N = op.n_dofs
    g = torch.Generator(device="cuda").manual_seed(0)
    T = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
    op.set_linearization(T, T)
    nq = op.n_cells * (a.degree + 1) ** 3
    if a.transport:
        x = op.support_points()
        hs = (0.5 + 0.5 * torch.tanh((x[:, 2] - 0.5) / 0.05)).contiguous()
        vel = torch.stack([torch.sin(3 * x[:, 1]), 0.5 + x[:, 2], -x[:, 0] * x[:, 1]]).contiguous()
        op.set_fields(hs, vel)
    if a.picard:
        x = torch.rand(N, dtype=torch.float32, device="cuda", generator=g)
        y = torch.empty_like(x)
        op.set_picard_tensor_cores(True)  # opt-in; exists for uniform boxes at FE_Q(3)
        for tc in ([True, False] if op.picard_tensor_cores else [False]):
            op.set_picard_tensor_cores(tc)
            for _ in range(3):
                op.vmult_picard_f32(y, x)
            torch.cuda.synchronize()
            # the verb also rebuilds the conductivity field and zeroes dst: time the operator
            # kernel alone with the library's own events around it
            op.set_timing(True)
            op.counters(reset=True)
            for _ in range(a.reps):
                op.vmult_picard_f32(y, x)
            torch.cuda.synchronize()
            c = op.counters(reset=True)
            op.set_timing(False)
            ms = c["vmult32_ms"] / max(c["vmult32_calls"], 1)
            alg = 2 * 4 * N + 4 * nq
            print(json.dumps({"degree": a.degree, "cells": a.cells, "operator": "picard_f32",
                              "kernel": "tensor-core" if tc else "cuda-core", "n_dofs": N,
                              "ms": ms, "gdofs": N / ms / 1e6, "alg_bytes": alg,
                              "alg_gbs": alg / ms / 1e6}), flush=True)
        return
    if a.solve:
        from meltpooldg_b200 import _lib as L
        op.distribute_constraints(T)
        H.JacobiPreconditioner(op).update()
        b = op.vmult(op.new_vector(), torch.rand(N, dtype=torch.float64, device="cuda",
                                                 generator=g))
        data = H.LinearSolverData(preconditioner_type=L.PRECOND_CHEBYSHEV_JACOBI_F32,
                                  cheb_degree=6, cheb_picard=True, max_iterations=3,
                                  rel_tolerance=1e-30)
        try:
            H.LinearSolver.solve(op, op.new_vector(), b, data, True)
        except H.ExcNoConvergence:
            pass
        torch.cuda.synchronize()
        print("solve done")
        return
    for dt in (["f64", "f32"] if a.dtype == "both" else [a.dtype]):
        ty = torch.float64 if dt == "f64" else torch.float32
        s = 8 if dt == "f64" else 4
        x = torch.rand(N, dtype=ty, device="cuda", generator=g)
        y = torch.empty_like(x)
        if a.transport:  # the first application after a new linearisation builds the fields
            op.set_linearization(T, T)
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        op.vmult(y, x)
        s1.record()
        torch.cuda.synchronize()
        first_ms = s0.elapsed_time(s1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.reps):
            op.vmult(y, x)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        tangent_fields = a.transport and a.law == 4 and a.degree <= (3 if dt == "f64" else 4)
        if tangent_fields:
            alg = s * N * 2 + 8 * s * nq + (7 * s * nq if a.perturb > 0 else 0)
        elif a.transport:
            alg = s * N * (2 + (2 if a.law == 4 else 0)) + 5 * s * nq + (7 * s * nq if a.perturb > 0 else 0)
        else:
            alg = s * N * (2 + (1 if a.law else 0)) + (7 * s * nq if a.perturb > 0 else 0)
        print(json.dumps({"degree": a.degree, "cells": a.cells, "perturb": a.perturb,
                          "law": a.law, "transport": a.transport, "dtype": dt,
                          "setup_ms": first_ms - ms if a.transport else None, "n_dofs": N, "ms": ms,
                          "gdofs": N / ms / 1e6, "alg_bytes": alg,
                          "alg_gbs": alg / ms / 1e6}), flush=True)


if __name__ == "__main__":
    main()
