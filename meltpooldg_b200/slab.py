"""Slab decomposition of the heat operator over ranks, one GPU per rank.

MeltPoolDG distributes its triangulation over MPI ranks and sums the contributions of DoFs on
partition boundaries with a ghost exchange (MatrixFree::loop with
LinearAlgebra::distributed::Vector::compress(add) / update_ghost_values, scratch_data.cpp:149-188);
dot products and norms are MPI_Allreduce'd. Here the structured box is split into z-slabs of
cells, one per rank (`mpdg_heat_create_slab`). A rank holds the global DoF planes
K = p z_begin .. p z_end; its first and last planes are shared with the neighbouring slabs.

Vectors are stored per rank as the local part including both shared planes, kept consistent
(equal values on both owners of a shared plane). After every assembly (operator application,
diagonal, residual) each rank adds its neighbours' partial sums of the shared planes: one plane
(n_x n_y values) sent to and received from each neighbour, over NCCL (`batch_isend_irecv` on the
device buffers) or, with a host backend (gloo), staged through host memory. Both owners compute
`mine + theirs`, and floating-point addition commutes, so the shared planes stay bitwise equal.
In dot products a shared plane is counted by the upper slab only. The cell integrals of the L2
norm are disjoint and need no weighting.

The solvers are Jacobi-preconditioned CG (deal.II SolverCG with ReductionControl, as
`LinearSolver::solve`) and the implicit step of HeatDiffuseOperation (predictor, history
commit, Jacobi update at the predicted state, Newton-Raphson). A CG iteration is one operator
application, one plane exchange and the library's fused stage kernels (`mpdg_heat_dcg_*`: the
vector updates with their partial dot products over the owned DoFs), with two all-reduces of
device buffers; the step lengths stay on the device, so the only host read per iteration is the
convergence test. Every branch that involves a collective is taken on a globally reduced value,
so all ranks take it.
"""
from __future__ import annotations

import math

import torch
import torch.distributed as dist

from . import _lib as L
from .heat import (ExcInvalidArgument, ExcNoConvergence, HeatDiffuseOperator, LinearSolverData,
                   NonlinearSolverData)


def slab_ranges(n_cells_z: int, world: int):
    """Balanced split of the z cell layers over the ranks: [(z_begin, z_end), ...]."""
    if world < 1 or n_cells_z < world:
        raise ExcInvalidArgument("need at least one cell layer per rank")
    base, extra = divmod(n_cells_z, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((z, z + n))
        z += n
    return out


class SlabExchange:
    """Sums the shared DoF planes of a slab vector with the neighbouring ranks."""

    def __init__(self, group=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.staged = dist.get_backend(group) != "nccl"

    def _peer(self, r):
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def add_shared_planes(self, v: torch.Tensor, plane: int):
        """v[:plane] += lower neighbour's last plane, v[-plane:] += upper neighbour's first."""
        if self.world == 1:
            return v
        lo = v[:plane]
        hi = v[v.numel() - plane:]
        sends, recvs = [], []
        if self.rank > 0:
            sends.append((self.rank - 1, lo.clone()))
            recvs.append((self.rank - 1, torch.empty_like(lo)))
        if self.rank < self.world - 1:
            sends.append((self.rank + 1, hi.clone()))
            recvs.append((self.rank + 1, torch.empty_like(hi)))
        if self.staged:
            sends = [(r, t.cpu()) for r, t in sends]
            recvs = [(r, t.cpu()) for r, t in recvs]
        ops = [dist.P2POp(dist.isend, t, self._peer(r), self.group) for r, t in sends]
        ops += [dist.P2POp(dist.irecv, t, self._peer(r), self.group) for r, t in recvs]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        for r, t in recvs:
            (lo if r < self.rank else hi).add_(t.to(v.device))
        return v

    def all_reduce_(self, t: torch.Tensor) -> torch.Tensor:
        """In-place sum over the ranks of a small tensor: on the device over NCCL, staged
        through host memory with a host backend (gloo)."""
        if self.world == 1:
            return t
        if self.staged and t.is_cuda:
            h = t.cpu()
            dist.all_reduce(h, group=self.group)
            t.copy_(h)
        else:
            dist.all_reduce(t, group=self.group)
        return t

    def sum(self, x: float) -> float:
        if self.world == 1:
            return float(x)
        dev = "cpu" if self.staged else torch.device("cuda", torch.cuda.current_device())
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, group=self.group)
        return float(t.item())


class SlabHeatOperator:
    """HeatDiffuseOperator on this rank's z-slab of the global box `mesh`."""

    def __init__(self, mesh: L.MeshDesc, exchange: SlabExchange, device: int = 0, op=None):
        self.x = exchange
        self.mesh = mesh
        self.ranges = slab_ranges(mesh.cells[2], exchange.world)
        self.z_begin, self.z_end = self.ranges[exchange.rank]
        self.op = op if op is not None else HeatDiffuseOperator(
            mesh, device, slab=(self.z_begin, self.z_end))
        p = mesh.degree
        self.plane = (p * mesh.cells[0] + 1) * (p * mesh.cells[1] + 1)
        self.k_begin = p * self.z_begin  # global index of the first local DoF plane
        self.n_dofs = self.op.n_dofs
        last = exchange.rank == exchange.world - 1
        self.n_owned = self.n_dofs if last else self.n_dofs - self.plane

    # vectors -----------------------------------------------------------------------------
    def new_vector(self):
        return self.op.new_vector()

    def local_part(self, v_global: torch.Tensor) -> torch.Tensor:
        """This rank's planes of a global vector."""
        a = self.k_begin * self.plane
        return v_global[a:a + self.n_dofs].contiguous()

    def dot(self, a, b) -> float:
        n = self.n_owned
        return self.x.sum(torch.dot(a[:n], b[:n]).item())

    def norm(self, a) -> float:
        return self.dot(a, a) ** 0.5

    def l2_norm(self, u) -> float:
        return self.x.sum(self.op.l2_norm(u) ** 2) ** 0.5

    # operator verbs --------------------------------------------------------------------
    def set_material(self, m):
        self.op.set_material(m)

    def reset_time_increment(self, dt):
        self.op.reset_time_increment(dt)

    def set_linearization(self, T, T_old=None):
        self.op.set_linearization(T, T_old)

    def distribute_constraints(self, u):
        return self.op.distribute_constraints(u)

    def vmult(self, dst, src):
        self.op.vmult(dst, src)
        return self.x.add_shared_planes(dst, self.plane)

    def compute_inverse_diagonal(self, inv):
        """diag(J) summed over the slabs, inverted with |d| > 1e-10 ? 1/d : 1."""
        self.op.compute_diagonal(inv)
        self.x.add_shared_planes(inv, self.plane)
        return self.op.invert_diagonal(inv)

    def create_rhs(self, dst, T_old, heat_source=None):
        """dst += -R(T_lin) summed over the slabs."""
        tmp = self.new_vector()
        self.op.create_rhs(tmp, T_old, heat_source)
        self.x.add_shared_planes(tmp, self.plane)
        dst.add_(tmp)
        return dst


def slab_cg(A: SlabHeatOperator, x, b, inv_diag, data: LinearSolverData) -> int:
    """Jacobi-preconditioned CG across the slabs (deal.II SolverCG, ReductionControl:
    |r| <= max(abs_tol, rel_tol |r_0|)). Returns the iteration count.

    Each iteration: Ap = J p with the shared planes summed; the fused stage kernels of the
    operator (dcg_dot, dcg_update, dcg_direction) with their partial sums all-reduced as
    device tensors; alpha = rz / pAp and beta = rz' / rz computed on the device. The host reads
    (r.r, p.Ap) once per iteration for the convergence and breakdown tests."""
    op, X, n = A.op, A.x, A.n_owned
    r, z, p, ax = A.new_vector(), A.new_vector(), A.new_vector(), A.new_vector()
    dev = b.device
    part = torch.zeros(2, dtype=torch.float64, device=dev)
    pap = torch.zeros(1, dtype=torch.float64, device=dev)
    alpha = torch.zeros(1, dtype=torch.float64, device=dev)
    beta = torch.zeros(1, dtype=torch.float64, device=dev)
    nonzero_x = X.sum(float(x.abs().max().item())) > 0  # the same branch on every rank
    if nonzero_x:
        A.vmult(ax, x)
    op.dcg_start(n, b, ax if nonzero_x else None, inv_diag, r, z, p, part)
    X.all_reduce_(part)
    rz = part[:1].clone()
    res = math.sqrt(max(float(part[1]), 0.0))
    tol = max(data.abs_tolerance, data.rel_tolerance * res)
    if res <= tol:
        return 0
    for it in range(1, data.max_iterations + 1):
        A.vmult(ax, p)
        op.dcg_dot(n, p, ax, pap)
        X.all_reduce_(pap)
        torch.div(rz, pap, out=alpha)
        op.dcg_update(n, x, r, z, p, ax, inv_diag, alpha, part)
        X.all_reduce_(part)
        rr, pAp = torch.cat([part[1:], pap]).tolist()  # the iteration's one host read
        if not pAp > 0.0:
            raise ExcNoConvergence("CG breakdown: p.Ap <= 0")
        res = math.sqrt(max(rr, 0.0))
        if res <= tol:
            return it
        torch.div(part[:1], rz, out=beta)
        rz.copy_(part[:1])
        op.dcg_direction(p, z, beta)
    raise ExcNoConvergence(f"CG: {data.max_iterations} iterations, residual {res:.3e}")


class SlabHeatOperation:
    """HeatDiffuseOperation::solve across the slabs (linear-extrapolation predictor,
    history commit, Jacobi update at the predicted state, Newton-Raphson with Jacobi-CG
    increment solves; heat_diffuse_operation.cpp:213-289)."""

    def __init__(self, A: SlabHeatOperator, linear: LinearSolverData = None,
                 nonlinear: NonlinearSolverData = None, predictor=L.PREDICTOR_LINEAR):
        self.A = A
        self.linear = linear or LinearSolverData()
        self.nonlinear = nonlinear or NonlinearSolverData()
        self.predictor = predictor
        self.T = A.new_vector()
        self.T_old = A.new_vector()
        self.heat_source = None
        self.dt_old = 0.0
        self.newton_iterations = 0
        self.linear_iterations = 0

    def set_initial_condition(self, T0_local):
        self.T.copy_(T0_local)
        self.A.distribute_constraints(self.T)

    def solve(self, dt: float):
        A = self.A
        if self.predictor == L.PREDICTOR_LINEAR and abs(self.dt_old) >= 1e-12:
            pred = self.T + (dt / self.dt_old) * (self.T - self.T_old)
        else:
            pred = self.T.clone()
        self.T_old.copy_(self.T)
        self.T.copy_(pred)
        A.distribute_constraints(self.T)
        A.reset_time_increment(dt)
        A.set_linearization(self.T, self.T_old)
        inv = A.compute_inverse_diagonal(A.new_vector())
        self.newton_iterations = self.linear_iterations = 0
        converged = False
        for i in range(self.nonlinear.max_nonlinear_iterations):
            rhs = A.create_rhs(A.new_vector(), self.T_old, self.heat_source)
            du = A.new_vector()
            self.linear_iterations += slab_cg(A, du, rhs, inv, self.linear)
            if (A.norm(rhs) < self.nonlinear.residual_tolerance and
                    A.norm(du) < self.nonlinear.field_correction_tolerance):
                converged = True
                break
            self.T.add_(du)
            A.distribute_constraints(self.T)
            A.set_linearization(self.T, self.T_old)
            self.newton_iterations = i + 1
        if not converged:
            raise ExcNoConvergence("Newton-Raphson did not converge")
        self.dt_old = float(dt)
        return self
