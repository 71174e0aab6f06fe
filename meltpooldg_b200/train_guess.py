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
    a = ap.parse_args()
    t0 = time.time()
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
