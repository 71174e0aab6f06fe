"""Benchmark: implicit heat steps of the nonlinear k(T) heat problem on B200.

Workload (one "step" = one implicit Euler step of the hot path): FE_Q(3) on the
unit cube with 128^3 cells (385^3 = 57,066,625 DoFs), k(T) = 1 + 0.5 T,
rho*cp = 1, dt = 5e-4, Dirichlet T = 0 on all faces, T0 = 0, a Gaussian source
of radius 0.05 at z = 0.95 moving along x at speed 1, one Newton linearisation
per step solved to |b - J T| <= 1e-8 |b|. The solvers run the same steps:
  plain    FP64 Jacobi-CG
  mixed    FP64 flexible CG with the FP32 p-multigrid V-cycle preconditioner
  cheb     FP64 flexible CG with the FP32 degree-6 Chebyshev-Jacobi preconditioner
  learned  the mixed solver started from the learned guess
`value` is the step throughput of the fastest one (named in "variant") in DoFs
advanced per second (whole job: summed over replicas when run with --gpus N > 1,
which runs independent replicas: the path has no data-parallel exchange on one
mesh). The CPU baseline and the reference arm run the oracle port (the reference's
plain FP64 Jacobi-CG step) on the same 128^3 workload, bounded to a few steps; the
first step's CPU solution is the FP64 reference of "error_vs_cpu_fp64".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Heat step time @1e-8 resid: learned+mixed vs plain FP64 CG; MF vmult GDoF/s"
DEGREE, CELLS, DT, K1 = 3, 128, 5e-4, 0.5
AMP, RADIUS, Z0, SPEED, X0 = 500.0, 0.05, 0.95, 1.0, 0.1
REL_TOL = 1e-8
CHEB_DEGREE = 6
REF_WARMUP, REF_STEPS = 1, 2  # CPU reference arm: bounded sample of the requested steps


def source_center(t):
    return (X0 + SPEED * t, 0.5, Z0)


def workload_config(cells):
    n = (DEGREE * cells + 1) ** 3
    return {
        "workload": f"implicit k(T) heat step, FE_Q({DEGREE}) unit cube {cells}^3 cells "
                    f"({n} DoFs), k=1+{K1}T, rho*cp=1, dt={DT}, Dirichlet 0, moving Gaussian "
                    f"source r={RADIUS} z={Z0} v={SPEED}, one linearisation, |b-JT|<={REL_TOL}|b|",
        "degree": DEGREE, "cells": [cells] * 3, "n_dofs": n,
        "l2_flush": "inputs larger than L2 (each FP64 vector is %.0f MB > 126 MB L2)" % (n * 8 / 1e6),
    }


# ---------------------------------------------------------------------------
# clock sampling
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU legs (oracle port: the reference's algorithm restated in C, OpenMP)
# ---------------------------------------------------------------------------
def cpu_step_sample(cells, steps, first=0, keep=None):
    """Implicit steps `first` .. `first + steps - 1` of the same problem with the oracle
    (plain FP64 Jacobi-CG, the reference's algorithm), from T0 = 0; the steps before
    `first` run untimed. Returns (DoFs/s, seconds, n_dofs, cores); with a dict `keep`, the
    solution after the first step is stored in keep["T1"]."""
    import numpy as np
    from oracle import oracle as O
    o = O.Oracle(DEGREE, (cells,) * 3)
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=K1), DT)
    T = np.zeros(o.n_dofs)
    T_old = np.zeros(o.n_dofs)
    dt_old = 0.0
    t0 = time.perf_counter()
    for s in range(first + steps):
        if s == first:
            t0 = time.perf_counter()
        t = (s + 1) * DT
        q = o.gaussian_source(AMP, source_center(t), RADIUS)
        Tg = o.linear_predictor(T, T_old, DT, dt_old)
        T_old, T = T, o.distribute(Tg)
        r = o.create_rhs(T, T_old, q)
        b = o.vmult(T, T, T_old) + r
        bn, rn = float(np.linalg.norm(b)), float(np.linalg.norm(r))
        if rn > 0.0:
            d, _, _ = o.cg(r, T_lin=T, T_old=T_old, rel_tol=REL_TOL * bn / rn, abs_tol=0.0)
            T = T + d
        if keep is not None and s == 0:
            keep["T1"] = T.copy()
        dt_old = DT
    sec = time.perf_counter() - t0
    return o.n_dofs * steps / sec, sec, o.n_dofs, os.cpu_count()


def run_reference(args):
    """The reference's algorithm (plain FP64 Jacobi-CG steps, the oracle port on all host
    cores) on the benchmark's own workload. A CPU step of the 128^3 mesh takes tens of
    seconds, so the run is a bounded sample: at most REF_WARMUP untimed and REF_STEPS timed
    steps of the requested W and K (stated in the line)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cells = args.cpu_cells
    warm, steps = min(args.warmup, REF_WARMUP), min(args.steps, REF_STEPS)
    rate, sec, n, cores = cpu_step_sample(cells, steps, first=warm)
    sample = (f"steps {warm}..{warm + steps - 1} of the workload on {cells}^3 cells ({n} DoFs) "
              f"after {warm} untimed, oracle port (OpenMP, {cores} threads); a bounded sample "
              f"of the requested --warmup {args.warmup} --steps {args.steps}")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "DoF/s",
            "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "steps_requested": args.steps, "warmup_requested": args.warmup,
            "ms_per_step": 1e3 * sec / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(cells), "parallelism": "CPU, rank 0 only",
            "cpu_baseline": {"value": rate, "unit": "DoF/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": rate, "unit": "DoF/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# multi-rank helpers (one process per GPU; each rank runs an independent replica)
# ---------------------------------------------------------------------------
def max_over_ranks(value, device, world):
    """The largest value over the ranks (device times: the slowest replica sets the
    job time); the value itself on a single rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gpu_local_cpus(dev_index):
    """CPUs of the GPU's own NUMA node (NVML's CPU affinity of the device), or None when it
    cannot be read. Pinned host buffers allocated while the process runs there are placed in
    that node's memory, next to the GPU's PCIe root, so host<->device copies do not cross the
    inter-socket link."""
    try:
        import pynvml
        from cuda.bindings import runtime as cudart
        err, bus = cudart.cudaDeviceGetPCIBusId(64, dev_index)
        if int(err) != 0:
            return None
        bus = bus.split(b"\0", 1)[0].decode()
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            words = pynvml.nvmlDeviceGetCpuAffinity(h, (os.cpu_count() + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * w + b for w, m in enumerate(words) for b in range(64) if (m >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def pinned_near_gpu(dev_index, n, count):
    """`count` pinned float64 host buffers of n values on the GPU's NUMA node (the process's
    CPU affinity is restored afterwards); plain pinned buffers when the node is unknown."""
    import torch
    local = gpu_local_cpus(dev_index)
    before = os.sched_getaffinity(0)
    try:
        if local:
            os.sched_setaffinity(0, local)
        bufs = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(count)]
        for b in bufs:
            b.zero_()  # first touch on this node
    finally:
        os.sched_setaffinity(0, before)
    return bufs, sorted(local) if local else None


def replica_throughput(world, n_dofs, steps, ms):
    """Whole-job DoFs advanced per second: every replica advances n_dofs per step."""
    return world * n_dofs * steps / (ms / 1e3)


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """dram bytes per launch of the dominant kernel from the committed ncu summary."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        return d
    except Exception:
        return {}


def run_mine(args):
    import torch
    import torch.distributed as dist

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200 import heat as H

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    cells = args.cells

    op = H.HeatDiffuseOperator(H.box_mesh(DEGREE, (cells,) * 3), device=local)
    op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=K1))
    N = op.n_dofs
    plain = H.HeatDiffuseOperation(op, H.LinearSolverData(rel_tolerance=REL_TOL,
                                                          abs_tolerance=0.0),
                                   predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    mg_data = dict(preconditioner_type=L.PRECOND_MG_F32, rel_tolerance=REL_TOL,
                   abs_tolerance=0.0, cheb_picard=True, cheb_eig_reuse=True)
    mixed = H.HeatDiffuseOperation(op, H.LinearSolverData(**mg_data),
                                   predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    cheb = H.HeatDiffuseOperation(op, H.LinearSolverData(
        preconditioner_type=L.PRECOND_CHEBYSHEV_JACOBI_F32, rel_tolerance=REL_TOL,
        abs_tolerance=0.0, cheb_degree=CHEB_DEGREE, cheb_picard=True, cheb_eig_reuse=True),
        predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    learned = H.HeatDiffuseOperation(op, H.LinearSolverData(**mg_data),
                                     predictor=L.PREDICTOR_LINEAR_DIRECTION,
                                     single_linearization=True)
    q = op.new_vector()
    mixed.heat_source = q
    cheb.heat_source = q
    plain.heat_source = q
    learned.heat_source = q
    model = None
    if not args.no_learned:
        from meltpooldg_b200 import learned as LG
        # network trained on 32^3-cell meshes (nodal spacing 1/96): stride 4 on 128^3 cells
        model = LG.GuessModel.load(os.path.join(ROOT, "meltpooldg_b200", "models",
                                                "heat_guess_p3_h96"),
                                   stride=(DEGREE * cells) // 96 if cells % 32 == 0 else 1,
                                   device=local)
        guess_buf = op.new_vector()
    stream = torch.cuda.current_stream(dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()

    def march(opn, first, count):
        its = []
        for s in range(first, first + count):
            op.gaussian_source(q, AMP, source_center((s + 1) * DT), RADIUS)
            if opn is learned:
                if s == 0:
                    opn.params.predictor = L.PREDICTOR_LINEAR
                else:
                    # the network's increment direction; the step starts its increment solve
                    # from the residual-minimising multiple of it
                    model.direction(op, opn.T, opn.T_old, q, DT, out=guess_buf)
                    opn.set_direction(guess_buf)
                    opn.params.predictor = L.PREDICTOR_LINEAR_DIRECTION
            st = opn.solve(DT)
            its.append(st.linear_iterations)
        return its

    def timed(opn, first, count, instrument=False):
        barrier()
        if instrument:
            op.set_timing(True)
            op.counters(reset=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        its = march(opn, first, count)
        e1.record(stream)
        barrier()
        ms = e0.elapsed_time(e1)
        cnt = None
        if instrument:
            cnt = op.counters(reset=True)
            op.set_timing(False)
        ms = max_over_ranks(ms, dev, world)
        return ms, its, cnt

    W, K = args.warmup, args.steps
    # mixed precision first: the headline timed region (clock sampling, launch count),
    # then K more steps with per-operator CUDA-event timing for the kernel shares
    march(mixed, 0, 1)
    first_step = {"mixed": mixed.T.clone()}  # compared with the CPU FP64 solution below
    march(mixed, 1, W - 1)
    T_W, T_old_W = mixed.T.clone(), mixed.T_old.clone()  # state before the timed steps
    clocks = Clocks(local) if rank == 0 else None
    op.counters(reset=True)
    ms_mixed, its_mixed, _ = timed(mixed, W, K)
    launches = int(op.counters(reset=True)["launches"])
    clk = clocks.stop() if clocks else None
    init_res = mixed.last_stats.initial_relative_residual
    T_mixed = mixed.T.clone()  # after step W+K-1, compared with the plain solver below
    ms_instr, _, cnt = timed(mixed, W + K, K, instrument=True)
    # Chebyshev-preconditioned mixed precision on the same steps
    ms_cheb = its_cheb = None
    if not args.no_cheb:
        march(cheb, 0, W)
        ms_cheb, its_cheb, _ = timed(cheb, W, K)
    # learned guess + mixed precision on the same steps
    ms_learned = its_learned = init_res_learned = None
    if model is not None:
        march(learned, 0, W)
        ms_learned, its_learned, _ = timed(learned, W, K)
        init_res_learned = learned.last_stats.initial_relative_residual
    # plain FP64 Jacobi-CG on the same steps
    ms_plain = its_plain = None
    if not args.no_plain:
        march(plain, 0, 1)
        first_step["plain"] = plain.T.clone()
        march(plain, 1, W - 1)
        ms_plain, its_plain, _ = timed(plain, W, K)
    err = None
    if not args.no_plain:
        diff = torch.linalg.vector_norm(T_mixed - plain.T).item()
        ref = torch.linalg.vector_norm(plain.T).item()
        err = {"rel_l2": diff / ref if ref > 0 else 0.0,
               "rel_max": ((T_mixed - plain.T).abs().max() / plain.T.abs().max()).item()}
        del T_mixed

    # e2e: host-buffer C-ABI steps. Headline: the history resident on the device as
    # HeatDiffuseOperation keeps it (loaded once before the timed steps), each step uploads
    # its host source and downloads the new T. Also reported: the stateless call that copies
    # T, T_old and the source in and T, T_old out every step.
    e2e = None
    if not args.no_e2e:
        import ctypes as C
        (hT, hTo, hq), numa_cpus = pinned_near_gpu(dev.index if dev.index is not None else 0, N, 3)
        prm = mixed.params
        first = W

        def host_source(step, dst):
            op.gaussian_source(q, AMP, source_center((step + 1) * DT), RADIUS)
            dst.copy_(q)

        hT.copy_(T_W)  # the headline's steps W .. W+K-1 again, from the same state
        hTo.copy_(T_old_W)
        H.check(op._L.mpdg_heat_load_history(op.h, C.c_void_p(hT.data_ptr()),
                                             C.c_void_p(hTo.data_ptr())))
        ms_res = 0.0
        for st in range(first, first + K):
            host_source(st, hq)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            stt = L.StepStats()
            H.check(op._L.mpdg_heat_time_step_resident(op.h, C.byref(prm), DT, DT,
                                                        C.c_void_p(hq.data_ptr()),
                                                        C.c_void_p(hT.data_ptr()),
                                                        C.byref(stt)))
            e1.record(stream)
            barrier()
            ms_res += e0.elapsed_time(e1)
        ms_res = max_over_ranks(ms_res, dev, world)
        hT.copy_(T_W)
        hTo.copy_(T_old_W)
        ms_e2e = 0.0
        for st in range(first, first + K):
            host_source(st, hq)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            stt = L.StepStats()
            H.check(op._L.mpdg_heat_time_step_host(op.h, C.byref(prm), DT, DT,
                                                    C.c_void_p(hT.data_ptr()),
                                                    C.c_void_p(hTo.data_ptr()),
                                                    C.c_void_p(hq.data_ptr()), C.byref(stt)))
            e1.record(stream)
            barrier()
            ms_e2e += e0.elapsed_time(e1)
        ms_e2e = max_over_ranks(ms_e2e, dev, world)
        e2e = {"value": replica_throughput(world, N, K, ms_res), "unit": "DoF/s",
               "h2d_bytes_per_step": N * 8, "d2h_bytes_per_step": N * 8,
               "ms_per_step": ms_res / K,
               "api": "mpdg_heat_time_step_resident (history resident on the device, loaded "
                      "once; per step: host source in, new T out, pinned buffers)",
               "host_buffers": ("pinned, allocated on the GPU's NUMA node (CPUs "
                                f"{numa_cpus[0]}-{numa_cpus[-1]})" if numa_cpus else
                                "pinned (GPU's NUMA node unknown)"),
               "stateless": {"value": replica_throughput(world, N, K, ms_e2e), "unit": "DoF/s",
                             "h2d_bytes_per_step": 3 * N * 8, "d2h_bytes_per_step": 2 * N * 8,
                             "ms_per_step": ms_e2e / K,
                             "api": "mpdg_heat_time_step_host (T, T_old, source in; T, T_old out)"}}
        del hT, hTo, hq

    # vmult throughput of the FP64 operator (MF vmult GDoF/s), CUDA events
    x = torch.rand(N, dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    for _ in range(3):
        op.vmult(y, x)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        op.vmult(y, x)
    e1.record(stream)
    barrier()
    vm_ms = e0.elapsed_time(e1) / 10

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0

    # roofline of the dominant kernel of the step. Its share comes from the instrumented
    # steps; its duration from REPS back-to-back launches on the last linearisation point
    # (inside a solve, launches issued after convergence return at once and would
    # dilute a per-launch average).
    hbm, hbm_kind = peaks()
    nq = op.n_cells * (DEGREE + 1) ** 3
    REPS = 20
    picard_dominant = cnt["vmult32_ms"] >= cnt["vmult64_ms"]
    if picard_dominant:
        # FP32 Picard operator of the preconditioner: src + dst + conductivity per q-point
        # (the operand in cell rows when the step's smoother kept its iterate there: the
        # algorithmic bytes stay those of the lexicographic vectors)
        kname = ("k_vmult_picard_tc<4>" if op.picard_tensor_cores
                 else "k_vmult2<4,float,affine,conductivity_field,cell_rows>"
                 if op.picard_cell_rows else "k_vmult2<4,float,affine,conductivity_field>")
        kms = cnt["vmult32_ms"]
        alg_bytes = 2 * 4 * N + 4 * nq
        xs = torch.rand(N, dtype=torch.float32, device=dev)
        ys = torch.empty_like(xs)
        if op.picard_cell_rows:
            rows = torch.empty(op.cell_rows_size(), dtype=torch.float32, device=dev)
            op.to_cell_rows_f32(rows, xs)
            run = lambda: op.vmult_picard_f32_rows(ys, rows)
        else:
            run = lambda: op.vmult_picard_f32(ys, xs)
    else:
        kname = "k_vmult2<4,double,affine,linear_k_tangent_fields>"
        kms = cnt["vmult64_ms"]
        alg_bytes = 3 * 8 * N  # src + dst + linearisation point
        xs = torch.rand(N, dtype=torch.float64, device=dev)
        ys = torch.empty_like(xs)
        run = lambda: op.vmult(ys, xs)
    for _ in range(3):
        run()
    barrier()
    op.set_timing(True)
    op.counters(reset=True)
    for _ in range(REPS):
        run()
    barrier()
    c2 = op.counters(reset=True)
    op.set_timing(False)
    key = "vmult32" if picard_dominant else "vmult64"
    per_launch_ms = c2[key + "_ms"] / max(c2[key + "_calls"], 1)
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    tr = profile_traffic().get(kname)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm, "peak_source": f"{hbm_kind} hbm_gbs",
                "traffic": tr, "algorithmic_bytes_per_launch": alg_bytes,
                "avg_launch_ms": per_launch_ms, "timed_launches": REPS,
                "share_of_step": kms / ms_instr,
                "note": "share from CUDA events around every operator launch of K further "
                        "steps; duration from back-to-back launches"}

    # CPU baseline (rank 0, one GPU): the oracle port's first step of the same workload; its
    # solution is the FP64 CPU solution the GPU solvers' first step is compared with
    cpu = cpu_err = None
    if not args.no_cpu and world == 1:
        keep = {}
        rate, sec, n, cores = cpu_step_sample(args.cpu_cells, args.cpu_steps, keep=keep)
        cpu = {"value": rate, "unit": "DoF/s", "cores": cores, "kind": "port",
               "sample": f"the first {args.cpu_steps} implicit step(s) of the workload on "
                         f"{args.cpu_cells}^3 cells ({n} DoFs), oracle port (plain FP64 "
                         f"Jacobi-CG, OpenMP), {sec:.1f} s"}
        if args.cpu_cells == cells:
            ref = torch.from_numpy(keep["T1"]).to(dev)
            rn, rm = torch.linalg.vector_norm(ref).item(), ref.abs().max().item()
            cpu_err = {"step": 1, "reference": "oracle FP64 Jacobi-CG on the host, |b-JT|<=1e-8|b|"}
            for name, T1 in first_step.items():
                cpu_err[name] = {"rel_l2": torch.linalg.vector_norm(T1 - ref).item() / rn,
                                 "rel_max": (T1 - ref).abs().max().item() / rm}
            del ref
    del first_step

    # headline: the fastest solver on these steps (named in "variant"); every variant's
    # time is reported beside it
    variants = {"mixed": ms_mixed, "cheb": ms_cheb, "plain": ms_plain,
                "learned+mixed": ms_learned}
    best = min((v, k) for k, v in variants.items() if v)
    best_ms, best_name = best
    line = {
        "metric": METRIC, "value": replica_throughput(world, N, K, best_ms), "unit": "DoF/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": best_ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "variant": best_name,
        "variant_note": {
            "mixed": "FP64 flexible CG + FP32 p-multigrid, linear-extrapolation predictor",
            "learned+mixed": "the mixed solver started from the learned guess",
            "cheb": "FP64 flexible CG + FP32 Chebyshev(6)",
            "plain": "FP64 Jacobi-CG"}[best_name],
        "dtype": ("f64 (outer flexible CG, k(T) tangent, residual) + f32 (p-multigrid "
                  "preconditioner" + ("; fine-level operator TF32 on the tensor cores, FP32 "
                                      "accumulation)" if op.picard_tensor_cores else ")"))
                 if best_name != "plain" else "f64",
        "data": "synthetic",
        "config": workload_config(cells), "parallelism": f"replicas x{world}",
        "mixed_ms_per_step": ms_mixed / K,
        "plain_fp64_ms_per_step": ms_plain / K if ms_plain else None,
        "speedup_mixed_vs_plain": (ms_plain / ms_mixed) if ms_plain else None,
        "cg_iterations_mixed": its_mixed, "cg_iterations_plain": its_plain,
        "cheb_mixed_ms_per_step": ms_cheb / K if ms_cheb else None,
        "cg_iterations_cheb_mixed": its_cheb,
        "initial_relative_residual_last_step": init_res,
        "learned_mixed_ms_per_step": ms_learned / K if ms_learned else None,
        "speedup_learned_mixed_vs_plain": (ms_plain / ms_learned) if (ms_plain and ms_learned) else None,
        "cg_iterations_learned_mixed": its_learned,
        "initial_relative_residual_last_step_learned": init_res_learned,
        "mixed_solver": {"outer": "FP64 flexible CG", "preconditioner":
                         "FP32 p-multigrid V-cycle: FE_Q(3) -> FE_Q(1) on 128^3 -> FE_Q(1) "
                         "on 64^3, 32^3, 16^3, 8^3, 4^3; Chebyshev-Jacobi smoothing (2 pre, 2+1 "
                         "post steps over [upper/8, upper]; 8 steps on the coarsest level); "
                         "Picard operators (k(T_lin) at the q-points) on every level; Lanczos "
                         "intervals reused across steps", "predictor": "linear extrapolation (learned: plus the network's increment direction, "
                                      "scaled to minimise the initial residual)",
                         "outer_operator": "FP64 k(T) tangent from k(T_lin), k1 grad(T_lin) "
                                           "fields built once per linearisation (their build "
                                           "is inside the timed step)",
                         "launches": "one CG iteration recorded per solve as a CUDA graph and "
                                     "replayed",
                         "cheb": f"FP32 Chebyshev-Jacobi degree {CHEB_DEGREE}, Picard operator"},
        "mixed_vs_plain_error": err,
        "error_vs_cpu_fp64": cpu_err,
        "vmult_fp64_gdofs": N / (vm_ms / 1e3) / 1e9, "vmult_fp64_ms": vm_ms,
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": launches, "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--cells", type=int, default=CELLS)
    ap.add_argument("--cpu-cells", type=int, default=CELLS)
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cheb", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_mine(args)


if __name__ == "__main__":
    sys.exit(main())
