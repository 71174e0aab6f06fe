"""Implicit k(T) heat steps on one configuration: per-step time and outer
iterations of the mixed-precision solver (FP64 flexible CG + FP32 p-multigrid) and
of plain FP64 Jacobi-CG on the same steps, and the difference of their fields.

  python bench_steps.py --degree 4 --cells 96 --perturb 0.2 \\
      --steps 6 --warmup 2

Problem: unit cube, k(T) = 1 + 0.5 T, rho cp = 1, dt = 5e-4, Dirichlet 0, T0 = 0, a
Gaussian source (amplitude 500, radius 0.05, z = 0.95) on a back-and-forth
multi-track scan (tracks along x at y = 0.3, 0.5, 0.7, alternating direction,
speed 1), one linearisation per step solved to |b - J T| <= 1e-8 |b|.

With --transport the step is a melt-pool-like one: the three-phase gas-liquid-solid law
(solidus 0.3, liquidus 0.5) on a heaviside of a flat melt-pool surface at z = 0.9, a
recirculating velocity field v = 0.2 (sin(pi x) cos(pi z), 0, -cos(pi x) sin(pi z)), and
the nonsymmetric tangent solved by the reference's default GMRES with Jacobi ("plain")
against GMRES with the FP32 Chebyshev-Jacobi preconditioner ("mixed", flexible GMRES).
"""
from __future__ import annotations

import argparse
import json

import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H

DT, AMP, RADIUS, Z0, SPEED = 5e-4, 500.0, 0.05, 0.95, 1.0


def scan(t):
    """Position on the multi-track path after time t (tracks of length 0.8)."""
    s = SPEED * t
    track = int(s // 0.8) % 3
    u = s - 0.8 * (s // 0.8)
    x = 0.1 + u if track % 2 == 0 else 0.9 - u
    return (x, (0.3, 0.5, 0.7)[track], Z0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--degree", type=int, default=4)
    ap.add_argument("--cells", type=int, default=96)
    ap.add_argument("--perturb", type=float, default=0.2)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--transport", action="store_true")
    ap.add_argument("--cheb-degree", type=int, default=6,
                    help="degree of the FP32 Chebyshev preconditioner of the --transport solve")
    a = ap.parse_args()
    op = H.HeatDiffuseOperator(H.box_mesh(a.degree, (a.cells,) * 3, perturb=a.perturb, seed=1))
    q = op.new_vector()
    if a.transport:
        op.set_material(H.material(law=L.LAW_GAS_LIQUID_SOLID, rho=1.0, cp=1.0, k=1.0,
                                   rho_s=1.0, cp_s=1.2, k_s=1.5, T_solidus=0.3, T_liquidus=0.5,
                                   rho_g=0.1, cp_g=1.0, k_g=0.05))
        x = op.support_points()
        hs = (0.5 + 0.5 * torch.tanh((0.9 - x[:, 2]) / 0.02)).contiguous()
        pi = torch.pi
        vel = torch.stack([0.2 * torch.sin(pi * x[:, 0]) * torch.cos(pi * x[:, 2]),
                           torch.zeros_like(x[:, 0]),
                           -0.2 * torch.cos(pi * x[:, 0]) * torch.sin(pi * x[:, 2])]).contiguous()
        op.set_fields(hs, vel)
        solvers = {"mixed": H.LinearSolverData(solver_type=L.SOLVER_GMRES,
                                               preconditioner_type=L.PRECOND_CHEBYSHEV_JACOBI_F32,
                                               cheb_degree=a.cheb_degree, rel_tolerance=1e-8,
                                               abs_tolerance=0.0, cheb_eig_reuse=True)}
        if not a.no_plain:
            solvers["plain"] = H.LinearSolverData(solver_type=L.SOLVER_GMRES, rel_tolerance=1e-8,
                                                  abs_tolerance=0.0)
    else:
        op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
        solvers = {"mixed": H.LinearSolverData(preconditioner_type=L.PRECOND_MG_F32,
                                               rel_tolerance=1e-8, abs_tolerance=0.0,
                                               cheb_picard=True, cheb_eig_reuse=True)}
        if not a.no_plain:
            solvers["plain"] = H.LinearSolverData(rel_tolerance=1e-8, abs_tolerance=0.0)
    out = {"degree": a.degree, "cells": a.cells, "perturb": a.perturb, "n_dofs": op.n_dofs,
           "steps": a.steps, "warmup": a.warmup, "transport": a.transport,
           "cheb_degree": a.cheb_degree if a.transport else None}
    fields = {}
    for name, data in solvers.items():
        opn = H.HeatDiffuseOperation(op, data, predictor=L.PREDICTOR_LINEAR,
                                     single_linearization=True)
        opn.heat_source = q
        its = []

        def step(s):
            op.gaussian_source(q, AMP, scan((s + 1) * DT), RADIUS)
            its.append(opn.solve(DT).linear_iterations)
        for s in range(a.warmup):
            step(s)
        torch.cuda.synchronize()
        its.clear()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in range(a.warmup, a.warmup + a.steps):
            step(s)
        e1.record()
        torch.cuda.synchronize()
        out[name] = {"ms_per_step": e0.elapsed_time(e1) / a.steps, "iterations": list(its)}
        fields[name] = opn.T.clone()
        del opn
    if "plain" in fields:
        d, r = fields["mixed"] - fields["plain"], fields["plain"]
        out["mixed_vs_plain"] = {
            "rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(r)),
            "rel_max": float(d.abs().max() / r.abs().max())}
        out["speedup"] = out["plain"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
