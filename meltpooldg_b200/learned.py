"""Learned initial guess for the implicit heat step.

A new predictor type next to MeltPoolDG's linear extrapolation
(include/meltpooldg/linear_algebra/predictor.hpp:122-154, predictor_data.hpp:9-20):
guess = LE + alpha * a * P(y), with LE = 2 T^n - T^{n-1}, y the output of a small
BF16 U-Net (libmpdg_heat.so, mpdg_unet_*) evaluated on the nodal grid sampled
every `stride` DoFs per direction, P the trilinear prolongation, a the RMS of
T^n - T^{n-1} (inputs and output are scaled by it) and alpha the step length that
minimises the residual of the guess (so it is never worse than LE). The solver
still iterates to the same tolerance, so the network only shortens CG.

Training data come from trajectories of the plain FP64 solver along seeded
random straight scan paths; training runs the library's own forward, backward
and Adam kernels on the GPU.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time
from dataclasses import dataclass

import torch

from . import _lib as L
from . import heat as H

DT, K1, AMP, RADIUS, Z0 = 5e-4, 0.5, 500.0, 0.05, 0.95


def _check(rc):
    if rc != L.OK:
        msg = L.load().mpdg_unet_last_error().decode() or L.last_error()
        raise H._EXC.get(rc, H.MpdgError)(f"[{rc}] {msg}")


class UNet:
    """The library's U-Net on an (nx, ny, nz) grid; tensors are CUDA float32."""

    def __init__(self, dims, seed=1, device=0):
        self._L = L.load()
        self.dims = tuple(int(d) for d in dims)
        self.device = torch.device("cuda", device)
        h = C.c_void_p()
        _check(self._L.mpdg_unet_create(*self.dims, int(seed), C.byref(h)))
        self.h = h
        n = C.c_int64()
        _check(self._L.mpdg_unet_n_params(h, C.byref(n)))
        self.n_params = int(n.value)
        self.n_points = self.dims[0] * self.dims[1] * self.dims[2]
        self.sync_stream()

    def sync_stream(self):
        with torch.cuda.device(self.device):
            s = torch.cuda.current_stream().cuda_stream
        _check(self._L.mpdg_unet_set_stream(self.h, C.c_void_p(s)))

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self._L.mpdg_unet_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def get_params(self):
        p = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        _check(self._L.mpdg_unet_get_params(self.h, p.data_ptr()))
        return p

    def set_params(self, p):
        p = p.to(self.device, torch.float32).contiguous()
        _check(self._L.mpdg_unet_set_params(self.h, p.data_ptr()))

    def forward(self, x):
        x = x.contiguous()
        y = torch.empty(self.n_points, dtype=torch.float32, device=self.device)
        _check(self._L.mpdg_unet_forward(self.h, x.data_ptr(), y.data_ptr()))
        return y

    def backward(self, grad_out):
        g = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        _check(self._L.mpdg_unet_backward(self.h, grad_out.contiguous().data_ptr(), g.data_ptr()))
        return g

    def train_step(self, x, target, lr):
        loss = C.c_double()
        _check(self._L.mpdg_unet_train_step(self.h, x.contiguous().data_ptr(),
                                            target.contiguous().data_ptr(), float(lr),
                                            C.byref(loss)))
        return float(loss.value)


# layer shapes (must match nn_unet.cu): (Cin, Cout) of the 15 convolutions
LAYERS = [(3, 16), (16, 16), (16, 32), (32, 32), (32, 48), (48, 48), (48, 64), (64, 64),
          (64, 48), (48, 48), (48, 32), (32, 32), (32, 16), (16, 16), (16, 1)]


def unpack(params):
    """Split the flat parameter vector into [(weight[Cout, Cin, 3, 3, 3], bias[Cout])]."""
    out, off = [], 0
    for ci, co in LAYERS:
        w = params[off:off + ci * co * 27].view(co, ci, 3, 3, 3)
        off += ci * co * 27
        b = params[off:off + co]
        off += co
        out.append((w, b))
    assert off == params.numel()
    return out


@dataclass
class GuessModel:
    """A trained network, the sampling stride and the temperature input scale."""
    stride: int = 1
    T_scale: float = 1.0
    net: UNet | None = None

    def guess(self, op: H.HeatDiffuseOperator, T, T_old, q, dt, out=None, line_search=True):
        """Guess for the next step from (T^n, T^{n-1}, q^{n+1}); returns (guess, alpha)."""
        out = op.new_vector() if out is None else out
        self.net.sync_stream()
        alpha = C.c_double()
        H.check(op._L.mpdg_heat_learned_guess(op.h, self.net.h, self.stride, T.data_ptr(),
                                               T_old.data_ptr(),
                                               None if q is None else q.data_ptr(), float(dt),
                                               float(self.T_scale), int(bool(line_search)),
                                               out.data_ptr(), C.byref(alpha)))
        return out, float(alpha.value)

    def direction(self, op: H.HeatDiffuseOperator, T, T_old, q, dt, out=None):
        """The network's increment direction a P(y) for PREDICTOR_LINEAR_DIRECTION (the step
        starts its increment solve from alpha times it, alpha minimising the residual)."""
        out = op.new_vector() if out is None else out
        self.net.sync_stream()
        H.check(op._L.mpdg_heat_learned_direction(op.h, self.net.h, self.stride, T.data_ptr(),
                                                   T_old.data_ptr(),
                                                   None if q is None else q.data_ptr(),
                                                   float(dt), float(self.T_scale),
                                                   out.data_ptr()))
        return out

    def save(self, path):
        p = self.net.get_params().cpu()
        torch.save({"params": p, "dims": self.net.dims, "T_scale": self.T_scale}, path + ".pt")
        with open(path + ".json", "w") as f:
            json.dump({"dims": list(self.net.dims), "T_scale": self.T_scale,
                       "n_params": self.net.n_params}, f, indent=1)

    @classmethod
    def load(cls, path, stride=1, device=0):
        d = torch.load(path + ".pt", map_location="cpu")
        net = UNet(d["dims"], device=device)
        net.set_params(d["params"])
        return cls(stride=stride, T_scale=float(d["T_scale"]), net=net)


def scan_path(rng: torch.Generator):
    """Straight scan segment: start in [0.1, 0.9]^2, random heading, speed 1."""
    u = torch.rand(3, generator=rng, dtype=torch.float64).tolist()
    x0, y0 = 0.1 + 0.8 * u[0], 0.1 + 0.8 * u[1]
    th = 2.0 * math.pi * u[2]
    return lambda t: (x0 + t * math.cos(th), y0 + t * math.sin(th), Z0)


def make_operator(cells, degree=3, device=0):
    op = H.HeatDiffuseOperator(H.box_mesh(degree, (cells,) * 3), device=device)
    op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=K1))
    return op


def generate(op, n_traj, n_steps, seed, stride=1, T_scale=0.1, amp=AMP, solver_tol=1e-10):
    """Trajectories of the plain FP64 solver along seeded random scan paths. Returns
    [(input[3 G], target[G])] on the sampled grid, normalised as the guess normalises
    them: inputs (T^n - T^{n-1})/a, dt q/a, T^n/T_scale and target
    (T^{n+1} - 2 T^n + T^{n-1})/a with a = RMS(T^n - T^{n-1})."""
    g = torch.Generator().manual_seed(seed)
    lin = H.LinearSolverData(rel_tolerance=solver_tol, abs_tolerance=0.0)
    dims = tuple((d - 1) // stride + 1 for d in op.dims)
    npts = dims[0] * dims[1] * dims[2]
    samples = []
    for _ in range(n_traj):
        path = scan_path(g)
        opn = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR,
                                     single_linearization=True)
        q = op.new_vector()
        opn.heat_source = q
        for s in range(n_steps):
            op.gaussian_source(q, amp, path((s + 1) * DT), RADIUS)
            T_n, T_nm1 = opn.T.clone(), opn.T_old.clone()
            a = float((T_n - T_nm1).pow(2).mean().sqrt())
            x = None
            if s > 0 and a > 0.0:
                x = torch.empty(3 * npts, dtype=torch.float32, device=op.device)
                sc = (C.c_double * 3)(a, a, T_scale)
                H.check(op._L.mpdg_heat_learned_input(op.h, stride, T_n.data_ptr(),
                                                      T_nm1.data_ptr(), q.data_ptr(), DT, sc,
                                                      x.data_ptr()))
            opn.solve(DT)
            if x is None:
                continue
            tgt = (opn.T - 2.0 * T_n + T_nm1).view(op.dims[2], op.dims[1], op.dims[0])
            tgt = tgt[::stride, ::stride, ::stride].contiguous().view(-1) / a
            samples.append((x, tgt.float().contiguous()))
    return samples


def train(net: UNet, samples, steps, lr=5e-4, seed=0, log_every=0):
    """Adam with a cosine learning-rate decay on the MSE; returns the loss history."""
    g = torch.Generator().manual_seed(seed)
    hist = []
    for it in range(steps):
        i = int(torch.randint(len(samples), (1,), generator=g))
        cur_lr = lr * 0.5 * (1.0 + math.cos(math.pi * it / steps))
        hist.append(net.train_step(samples[i][0], samples[i][1], cur_lr))
        if log_every and it % log_every == 0:
            print(f"step {it} loss {hist[-1]:.4e}", flush=True)
    return hist


def train_streaming(op, net: UNet, n_traj, n_steps, seed, lr=5e-4, T_scale=0.1, amp=AMP,
                    solver_tol=1e-10, stride=1, passes=1, log_every=0, max_seconds=None):
    """Train while the trajectories are generated (the samples of a large grid do not fit in
    memory: 115 MB each on 193^3): for each seeded straight scan path, every step's sample
    (the normalised inputs and target of `generate`) takes `passes` Adam steps right after the
    solver produced it (FP64 CG with the FP32 p-multigrid to `solver_tol`). A cosine learning-rate
    decay over all planned steps. Returns (losses, samples seen, trajectories done)."""
    g = torch.Generator().manual_seed(seed)
    lin = H.LinearSolverData(preconditioner_type=L.PRECOND_MG_F32, rel_tolerance=solver_tol,
                             abs_tolerance=0.0, cheb_picard=True, cheb_eig_reuse=True)
    dims = tuple((d - 1) // stride + 1 for d in op.dims)
    npts = dims[0] * dims[1] * dims[2]
    total = max(1, n_traj * (n_steps - 1) * passes)
    x = torch.empty(3 * npts, dtype=torch.float32, device=op.device)
    hist, seen, it = [], 0, 0
    t0 = time.time()
    done = 0
    for _ in range(n_traj):
        path = scan_path(g)
        opn = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR,
                                     single_linearization=True)
        q = op.new_vector()
        opn.heat_source = q
        for s in range(n_steps):
            op.gaussian_source(q, amp, path((s + 1) * DT), RADIUS)
            T_n, T_nm1 = opn.T.clone(), opn.T_old.clone()
            a = float((T_n - T_nm1).pow(2).mean().sqrt())
            use = s > 0 and a > 0.0
            if use:
                sc = (C.c_double * 3)(a, a, T_scale)
                H.check(op._L.mpdg_heat_learned_input(op.h, stride, T_n.data_ptr(),
                                                      T_nm1.data_ptr(), q.data_ptr(), DT, sc,
                                                      x.data_ptr()))
            opn.solve(DT)
            if not use:
                continue
            tgt = (opn.T - 2.0 * T_n + T_nm1).view(op.dims[2], op.dims[1], op.dims[0])
            tgt = (tgt[::stride, ::stride, ::stride].contiguous().view(-1) / a).float()
            for _ in range(passes):
                cur = lr * 0.5 * (1.0 + math.cos(math.pi * min(it, total) / total))
                hist.append(net.train_step(x, tgt, cur))
                it += 1
            seen += 1
            if log_every and seen % log_every == 0:
                print(f"sample {seen} loss {hist[-1]:.4e} {time.time() - t0:.0f} s", flush=True)
        done += 1
        del opn
        if max_seconds is not None and time.time() - t0 > max_seconds:
            break
    return hist, seen, done


def evaluate(op, model, seeds, n_steps, mg=True):
    """Held-out scan paths: per step the outer iterations and the device time (CUDA events) of
    the step to |b - J T| <= 1e-8 |b|, with the linear extrapolation alone and with the
    network's increment direction (its forward pass included in the learned step's time)."""
    lin = H.LinearSolverData(preconditioner_type=L.PRECOND_MG_F32 if mg else L.PRECOND_JACOBI,
                             rel_tolerance=1e-8, abs_tolerance=0.0, cheb_picard=True,
                             cheb_eig_reuse=True)
    out = {}
    for name in ("extrapolation", "learned"):
        its, ms = [], []
        for sd in seeds:
            path = scan_path(torch.Generator().manual_seed(sd))
            opn = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR,
                                         single_linearization=True)
            q = op.new_vector()
            opn.heat_source = q
            d = op.new_vector()
            for s in range(n_steps):
                op.gaussian_source(q, AMP, path((s + 1) * DT), RADIUS)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                if name == "learned" and s > 0:
                    model.direction(op, opn.T, opn.T_old, q, DT, out=d)
                    opn.set_direction(d)
                    opn.params.predictor = L.PREDICTOR_LINEAR_DIRECTION
                st = opn.solve(DT)
                e1.record()
                torch.cuda.synchronize()
                if s > 0:
                    its.append(st.linear_iterations)
                    ms.append(e0.elapsed_time(e1))
            del opn
        out[name] = {"iterations": its, "mean_iterations": sum(its) / len(its),
                     "mean_ms": sum(ms) / len(ms)}
    return out
