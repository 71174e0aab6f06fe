"""Forward, backward and training-step times of the learned-guess network on an (nx, ny, nz)
grid.

    python bench_unet.py --dims 97 97 97 [--reps 10]

prints one JSON line with the CUDA-event time per forward (tensor-core convolutions, or the
CUDA-core ones with MPDG_UNET_TC=0), per backward (data gradients on the tensor cores, or on
the CUDA cores with MPDG_UNET_TC_BWD=0; weight gradients on the CUDA cores), per training step
(forward + backward + Adam) and the nominal FLOPs of the convolutions."""
import argparse
import json
import os

import torch

from meltpooldg_b200 import learned as LG


def conv_flops(dims):
    """2 * 27 * Ci * Co multiply-adds per output point, summed over the layers."""
    sizes = [tuple(dims)]
    for _ in range(3):
        sizes.append(tuple((d + 1) // 2 for d in sizes[-1]))
    pts = [s[0] * s[1] * s[2] for s in sizes]
    level = [0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0, 0]
    return sum(2 * 27 * ci * co * pts[lv] for (ci, co), lv in zip(LG.LAYERS, level))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=3, default=[97, 97, 97])
    ap.add_argument("--reps", type=int, default=10)
    a = ap.parse_args()
    n = a.dims[0] * a.dims[1] * a.dims[2]
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(3 * n, device="cuda", generator=g)
    net = LG.UNet(tuple(a.dims), seed=1)
    for _ in range(3):
        net.forward(x)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        y = net.forward(x)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    gy = torch.randn(n, device="cuda", generator=g)
    for _ in range(2):
        net.backward(gy)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.reps):
        gp = net.backward(gy)
    e1.record()
    torch.cuda.synchronize()
    ms_bwd = e0.elapsed_time(e1) / a.reps
    t = torch.randn(n, device="cuda", generator=g)
    for _ in range(2):
        net.train_step(x, t, 1e-4)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.reps):
        net.train_step(x, t, 1e-4)
    e1.record()
    torch.cuda.synchronize()
    ms_train = e0.elapsed_time(e1) / a.reps
    fl = conv_flops(a.dims)
    tc_bwd = os.environ.get("MPDG_UNET_TC") != "0" and os.environ.get("MPDG_UNET_TC_BWD") != "0"
    print(json.dumps({"dims": a.dims, "path": "cuda-core" if os.environ.get("MPDG_UNET_TC") == "0"
                      else "tensor-core",
                      "data_gradient": "tensor-core" if tc_bwd else "cuda-core",
                      "forward_ms": ms, "backward_ms": ms_bwd, "train_step_ms": ms_train,
                      "conv_gflop": fl / 1e9, "conv_tflops": fl / ms / 1e9,
                      "out_norm": float(y.norm()), "grad_norm": float(gp.norm())}), flush=True)


if __name__ == "__main__":
    main()
