"""The slab decomposition's host logic on CPU: gloo ranks, each with a z-slab of a Q1 box,
exchange their shared planes, count them once in dot products and reproduce the whole
mesh's operator application, diagonal, residual, CG solution and implicit steps.

The per-rank operator here is a small assembled Q1 operator written for this test
(M/dt + k K with the exact element matrices of an axis-aligned box cell, Dirichlet rows
zeroed), standing in for the CUDA slab handles so that the ranks run without a GPU; the
CUDA slabs themselves are tested in test_gpu_slab.py.
"""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from meltpooldg_b200 import heat as H
from meltpooldg_b200 import slab as S


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class BoxQ1:
    """Assembled Q1 operator M/dt + k K on the cells z in [z0, z1) of a box mesh."""

    def __init__(self, cells, hi, z0, z1, dirichlet, k=1.3, dt=0.05):
        m = [cells[0], cells[1], z1 - z0]
        h = [hi[e] / cells[e] for e in range(3)]
        nd = [m[0] + 1, m[1] + 1, m[2] + 1]
        self.n_dofs = nd[0] * nd[1] * nd[2]
        mass = [torch.tensor([[2.0, 1.0], [1.0, 2.0]], dtype=torch.float64) * (h[e] / 6)
                for e in range(3)]
        stiff = [torch.tensor([[1.0, -1.0], [-1.0, 1.0]], dtype=torch.float64) / h[e]
                 for e in range(3)]

        def kron3(a, b, c):  # z, y, x factors -> lexicographic (x fastest) 8x8
            return torch.kron(torch.kron(a, b), c)
        Me = kron3(mass[2], mass[1], mass[0])
        Ke = (kron3(stiff[2], mass[1], mass[0]) + kron3(mass[2], stiff[1], mass[0]) +
              kron3(mass[2], mass[1], stiff[0]))
        M = torch.zeros(self.n_dofs, self.n_dofs, dtype=torch.float64)
        K = torch.zeros_like(M)
        for cz in range(m[2]):
            for cy in range(m[1]):
                for cx in range(m[0]):
                    idx = torch.tensor([(cx + a) + nd[0] * ((cy + b) + nd[1] * (cz + c))
                                        for c in (0, 1) for b in (0, 1) for a in (0, 1)])
                    M[idx[:, None], idx[None, :]] += Me
                    K[idx[:, None], idx[None, :]] += Ke
        con = torch.zeros(self.n_dofs, dtype=torch.bool)
        I = torch.arange(self.n_dofs)
        i, j, kk = I % nd[0], (I // nd[0]) % nd[1], I // (nd[0] * nd[1])
        if dirichlet:
            con |= (i == 0) | (i == nd[0] - 1) | (j == 0) | (j == nd[1] - 1)
            con |= (kk == 0) & (z0 == 0)
            con |= (kk == nd[2] - 1) & (z1 == cells[2])
        self.con = con
        self.M, self.K, self.k, self.dt = M, K, k, dt
        self.T = self.To = None

    def new_vector(self):
        return torch.zeros(self.n_dofs, dtype=torch.float64)

    def _J(self):
        return self.M / self.dt + self.k * self.K

    def vmult(self, dst, src):
        s = torch.where(self.con, torch.zeros_like(src), src)
        dst.copy_(self._J() @ s)
        dst[self.con] = 0.0
        return dst

    def compute_diagonal(self, d):
        d.copy_(torch.diagonal(self._J()))
        d[self.con] = 0.0
        return d

    def create_rhs(self, dst, T_old, q=None):
        r = -(self.M @ (self.T - T_old) / self.dt + self.k * (self.K @ self.T))
        if q is not None:
            r += self.M @ q
        r[self.con] = 0.0
        dst.add_(r)
        return dst

    def distribute_constraints(self, u):
        u[self.con] = 0.0
        return u

    def l2_norm(self, u):
        return float(u @ (self.M @ u)) ** 0.5

    def set_material(self, m):
        pass

    # the CG stage kernels of the library (mpdg_heat_dcg_*), same semantics
    def invert_diagonal(self, d):
        ok = d.abs() > 1e-10
        d.copy_(torch.where(ok, 1.0 / torch.where(ok, d, torch.ones_like(d)), torch.ones_like(d)))
        return d

    def dcg_start(self, n_owned, b, Ax, D, r, z, p, partial):
        r.copy_(b if Ax is None else b - Ax)
        torch.mul(D, r, out=z)
        p.copy_(z)
        partial[0] = r[:n_owned] @ z[:n_owned]
        partial[1] = r[:n_owned] @ r[:n_owned]

    def dcg_dot(self, n_owned, a, b, partial):
        partial[0] = a[:n_owned] @ b[:n_owned]

    def dcg_update(self, n_owned, x, r, z, p, Ap, D, alpha, partial):
        x.add_(alpha * p)
        r.sub_(alpha * Ap)
        torch.mul(D, r, out=z)
        partial[0] = r[:n_owned] @ z[:n_owned]
        partial[1] = r[:n_owned] @ r[:n_owned]

    def dcg_direction(self, p, z, beta):
        p.mul_(beta).add_(z)

    def reset_time_increment(self, dt):
        self.dt = dt

    def set_linearization(self, T, T_old=None):
        self.T, self.To = T, T_old


CELLS, HI = (3, 2, 7), (1.0, 0.8, 1.4)


def _mesh():
    return H.box_mesh(1, CELLS, (0, 0, 0), HI)


class _OneRank:
    """The exchange of a one-rank run (no collectives)."""
    rank, world, staged, group = 0, 1, True, None

    def add_shared_planes(self, v, plane):
        return v

    def sum(self, x):
        return float(x)

    def all_reduce_(self, t):
        return t


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        x = S.SlabExchange()
        z0, z1 = S.slab_ranges(CELLS[2], world)[rank]
        A = S.SlabHeatOperator(_mesh(), x, op=BoxQ1(CELLS, HI, z0, z1, True))
        G = BoxQ1(CELLS, HI, 0, CELLS[2], True)  # the whole mesh on every rank
        g = torch.Generator().manual_seed(5)
        src = torch.rand(G.n_dofs, dtype=torch.float64, generator=g)
        T = G.distribute_constraints(torch.rand(G.n_dofs, dtype=torch.float64, generator=g))
        To = torch.rand(G.n_dofs, dtype=torch.float64, generator=g)
        q = torch.rand(G.n_dofs, dtype=torch.float64, generator=g)
        res = {}
        # operator verbs
        res["vmult"] = (A.vmult(A.new_vector(), A.local_part(src)) -
                        A.local_part(G.vmult(G.new_vector(), src))).abs().max().item()
        inv = A.compute_inverse_diagonal(A.new_vector())
        d = G.compute_diagonal(G.new_vector())
        ginv = torch.where(d.abs() > 1e-10, 1 / torch.where(d.abs() > 1e-10, d, 1.0), 1.0)
        res["diag"] = (inv - A.local_part(ginv)).abs().max().item()
        A.set_linearization(A.local_part(T), A.local_part(To))
        G.set_linearization(T, To)
        res["rhs"] = (A.create_rhs(A.new_vector(), A.local_part(To), A.local_part(q)) -
                      A.local_part(G.create_rhs(G.new_vector(), To, q))).abs().max().item()
        res["dot"] = abs(A.dot(A.local_part(src), A.local_part(q)) - float(src @ q))
        res["l2"] = abs(A.l2_norm(A.local_part(T)) - G.l2_norm(T))
        # CG on the slabs vs a dense solve of the whole mesh
        b = G.create_rhs(G.new_vector(), To, q)
        x_loc = A.new_vector()
        its = S.slab_cg(A, x_loc, A.local_part(b), inv,
                        H.LinearSolverData(rel_tolerance=1e-13, abs_tolerance=0.0))
        free = ~G.con
        xg = torch.zeros(G.n_dofs, dtype=torch.float64)
        xg[free] = torch.linalg.solve(G._J()[free][:, free], b[free])
        res["cg"] = (x_loc - A.local_part(xg)).abs().max().item() / xg.abs().max().item()
        res["cg_its"] = its
        # three implicit steps: slabs vs the whole mesh on one rank
        lin = H.LinearSolverData(rel_tolerance=1e-13, abs_tolerance=0.0)
        nl = H.NonlinearSolverData(residual_tolerance=1e-9)
        op_s = S.SlabHeatOperation(A, lin, nl)
        op_s.set_initial_condition(A.local_part(T))
        op_s.heat_source = A.local_part(q)
        op_g = S.SlabHeatOperation(S.SlabHeatOperator(_mesh(), _OneRank(), op=G), lin, nl)
        op_g.set_initial_condition(T)
        op_g.heat_source = q
        for _ in range(3):
            op_s.solve(0.05)
            op_g.solve(0.05)
        res["steps"] = ((op_s.T - A.local_part(op_g.T)).abs().max().item() /
                        op_g.T.abs().max().item())
        # shared planes are bitwise equal on both owners
        top = op_s.T[op_s.T.numel() - A.plane:].clone()
        bottom = op_s.T[:A.plane].clone()
        et = [torch.zeros_like(top) for _ in range(world)]
        eb = [torch.zeros_like(bottom) for _ in range(world)]
        dist.all_gather(et, top)
        dist.all_gather(eb, bottom)
        res["shared_equal"] = all(torch.equal(et[r], eb[r + 1]) for r in range(world - 1))
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_ranks_reproduce_the_whole_mesh(world):
    with mp.get_context("spawn").Manager() as m:  # no fork of this process
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True,
                           start_method="spawn")
        out = dict(out)
    assert sorted(out) == list(range(world))
    for r, res in out.items():
        assert res["vmult"] <= 1e-12, (r, res)
        assert res["diag"] <= 1e-12, (r, res)
        assert res["rhs"] <= 1e-12, (r, res)
        assert res["dot"] <= 1e-12 and res["l2"] <= 1e-12, (r, res)
        assert res["cg"] <= 1e-10 and res["cg_its"] > 0, (r, res)
        assert res["steps"] <= 1e-10, (r, res)
        assert res["shared_equal"], (r, res)
    assert len({res["cg_its"] for res in out.values()}) == 1


def test_slab_ranges():
    assert S.slab_ranges(7, 2) == [(0, 4), (4, 7)]
    assert S.slab_ranges(6, 3) == [(0, 2), (2, 4), (4, 6)]
    with pytest.raises(H.ExcInvalidArgument):
        S.slab_ranges(2, 3)
