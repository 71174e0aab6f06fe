"""Train the learned-guess network on trajectories of the plain FP64 solver.

  python -m meltpooldg_b200.train_guess --cells 32 --traj 16 --steps 20 --iters 2000 \
      --out meltpooldg_b200/models/heat_guess_p3_h96

The network runs on the nodal grid of a FE_Q(3) mesh with `cells`^3 cells; a mesh
refined k times per direction uses it with stride k (same nodal spacing).
"""
from __future__ import annotations

import argparse
import json
import time

import torch

from . import learned as LG


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=32)
    ap.add_argument("--traj", type=int, default=16)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--iters", type=int, default=2000)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--T-scale", type=float, default=0.1)
    ap.add_argument("--out", default="meltpooldg_b200/models/heat_guess_p3_h96")
    ap.add_argument("--stream", action="store_true",
                    help="train while generating (grids too large to keep the samples), then "
                         "evaluate on held-out seeds")
    ap.add_argument("--passes", type=int, default=1)
    ap.add_argument("--eval-seeds", type=int, nargs="*", default=[1001, 1002, 1003, 1004])
    ap.add_argument("--eval-steps", type=int, default=50)
    ap.add_argument("--max-minutes", type=float, default=None)
    a = ap.parse_args()
    t0 = time.time()
    if a.stream:
        op = LG.make_operator(a.cells)
        net = LG.UNet(op.dims, seed=a.seed)
        hist, seen, done = LG.train_streaming(
            op, net, a.traj, a.steps, a.seed, lr=a.lr, T_scale=a.T_scale, passes=a.passes,
            log_every=200, max_seconds=None if a.max_minutes is None else 60 * a.max_minutes)
        t1 = time.time()
        model = LG.GuessModel(stride=1, T_scale=a.T_scale, net=net)
        model.save(a.out)
        ev = LG.evaluate(op, model, a.eval_seeds, a.eval_steps)
        print(json.dumps({"cells": a.cells, "grid": list(op.dims), "trajectories": done,
                          "samples": seen, "train_s": t1 - t0, "eval_s": time.time() - t1,
                          "loss_first50": sum(hist[:50]) / max(1, len(hist[:50])),
                          "loss_last100": sum(hist[-100:]) / max(1, len(hist[-100:])),
                          "held_out": ev, "out": a.out}), flush=True)
        return
    op = LG.make_operator(a.cells)
    data = LG.generate(op, a.traj, a.steps, seed=a.seed, T_scale=a.T_scale)
    t1 = time.time()
    net = LG.UNet(op.dims, seed=a.seed)
    hist = LG.train(net, data, a.iters, lr=a.lr, seed=a.seed)
    torch.cuda.synchronize()
    model = LG.GuessModel(stride=1, T_scale=a.T_scale, net=net)
    model.save(a.out)
    print(json.dumps({"samples": len(data), "generate_s": t1 - t0, "train_s": time.time() - t1,
                      "loss_first50": sum(hist[:50]) / 50, "loss_last100": sum(hist[-100:]) / 100,
                      "out": a.out}), flush=True)


if __name__ == "__main__":
    main()
