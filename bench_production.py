"""Production run: 200 implicit k(T) steps on a deformed FE_Q(4) mesh, the learned guess with
the FP32 preconditioner against plain FP64 CG, in lock-step on one GPU.

  python bench_production.py [--steps 200] [--every 20] [--cells 96] [--degree 4]

Problem: unit cube, interior vertices perturbed by up to 0.2 h (seeded), FE_Q(4) on 96^3 cells
(385^3 = 57,066,625 DoFs), k(T) = 1 + 0.5 T, rho cp = 1, dt = 5e-4, Dirichlet 0, T0 = 0, a
Gaussian source (amplitude 500, radius 0.05, z = 0.95) on a seeded back-and-forth multi-track
scan (tracks along x, alternating direction, at seeded y positions, speed 1), one linearisation
per step solved to |b - J T| <= 1e-8 |b|. Three solvers advance the same steps:
  plain    FP64 Jacobi-CG (the reference's algorithm): the FP64 solution
  mixed    FP64 flexible CG + FP32 p-multigrid, linear-extrapolation predictor
  learned  the mixed solver with the learned increment direction
Every `--every` steps the L2 and max relative differences of mixed and learned against plain
are recorded. Prints one JSON line: per-step device times (CUDA events) and CG iterations of
each solver, the error series, and the means.
"""
from __future__ import annotations

import argparse
import json
import os

import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H

HERE = os.path.dirname(os.path.abspath(__file__))
DT, AMP, RADIUS, Z0, SPEED, TRACK = 5e-4, 500.0, 0.05, 0.95, 1.0, 0.8


def scan_path(seed: int):
    """Back-and-forth multi-track scan: tracks of length 0.8 along x (alternating direction),
    at y positions drawn from [0.2, 0.8] with a seeded generator."""
    g = torch.Generator().manual_seed(seed)
    ys = (0.2 + 0.6 * torch.rand(64, generator=g, dtype=torch.float64)).tolist()

    def at(t):
        s = SPEED * t
        k = int(s // TRACK)
        u = s - TRACK * k
        x = 0.1 + u if k % 2 == 0 else 0.9 - u
        return (x, ys[k % len(ys)], Z0)
    return at


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--degree", type=int, default=4)
    ap.add_argument("--cells", type=int, default=96)
    ap.add_argument("--perturb", type=float, default=0.2)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--every", type=int, default=20)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--no-learned", action="store_true")
    a = ap.parse_args()

    op = H.HeatDiffuseOperator(H.box_mesh(a.degree, (a.cells,) * 3, perturb=a.perturb, seed=1))
    op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
    N = op.n_dofs
    mg = dict(preconditioner_type=L.PRECOND_MG_F32, rel_tolerance=1e-8, abs_tolerance=0.0,
              cheb_picard=True, cheb_eig_reuse=True)
    ops = {"plain": H.HeatDiffuseOperation(op, H.LinearSolverData(rel_tolerance=1e-8,
                                                                   abs_tolerance=0.0),
                                           predictor=L.PREDICTOR_LINEAR,
                                           single_linearization=True),
           "mixed": H.HeatDiffuseOperation(op, H.LinearSolverData(**mg),
                                           predictor=L.PREDICTOR_LINEAR,
                                           single_linearization=True)}
    model = None
    stride = (op.dims[0] - 1) // 96 if (op.dims[0] - 1) % 96 == 0 else 0
    if not a.no_learned and stride > 0:
        from meltpooldg_b200 import learned as LG
        model = LG.GuessModel.load(os.path.join(HERE, "meltpooldg_b200", "models",
                                                "heat_guess_p3_h96"), stride=stride)
        ops["learned"] = H.HeatDiffuseOperation(op, H.LinearSolverData(**mg),
                                                predictor=L.PREDICTOR_LINEAR,
                                                single_linearization=True)
        direction = op.new_vector()
    q = op.new_vector()
    for opn in ops.values():
        opn.heat_source = q
    path = scan_path(a.seed)
    ms = {k: [] for k in ops}
    its = {k: [] for k in ops}
    errors = []
    for s in range(a.steps):
        op.gaussian_source(q, AMP, path((s + 1) * DT), RADIUS)
        for name, opn in ops.items():
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            if name == "learned" and s > 0:
                model.direction(op, opn.T, opn.T_old, q, DT, out=direction)
                opn.set_direction(direction)
                opn.params.predictor = L.PREDICTOR_LINEAR_DIRECTION
            st = opn.solve(DT)
            e1.record()
            torch.cuda.synchronize()
            ms[name].append(e0.elapsed_time(e1))
            its[name].append(st.linear_iterations)
        if (s + 1) % a.every == 0:
            ref = ops["plain"].T
            rn, rm = torch.linalg.vector_norm(ref).item(), ref.abs().max().item()
            row = {"step": s + 1, "T_max": rm}
            for name in ops:
                if name == "plain":
                    continue
                d = ops[name].T - ref
                row[name] = {"rel_l2": torch.linalg.vector_norm(d).item() / rn,
                             "rel_max": d.abs().max().item() / rm}
            errors.append(row)
    mean = {k: sum(v[1:]) / max(len(v) - 1, 1) for k, v in ms.items()}  # step 1 holds set-up
    out = {"config": {"degree": a.degree, "cells": a.cells, "perturb": a.perturb, "n_dofs": N,
                      "steps": a.steps, "dt": DT, "law": "k = 1 + 0.5 T", "scan_seed": a.seed,
                      "learned_stride": stride if model is not None else None},
           "mean_ms_per_step_after_first": mean,
           "speedup_vs_plain": {k: mean["plain"] / v for k, v in mean.items() if k != "plain"},
           "mean_iterations": {k: sum(v) / len(v) for k, v in its.items()},
           "errors_vs_plain_fp64": errors, "ms_per_step": ms, "iterations": its}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
