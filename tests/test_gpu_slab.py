"""CUDA slab handles across ranks: two processes on one GPU, each with its z-slab of the
mesh (mpdg_heat_create_slab), exchanging the shared planes through host-staged gloo
collectives (no kernel waits on another rank). Their operator application, inverse diagonal,
residual, L2 norm and implicit steps reproduce the whole mesh's on one handle."""
import os
import socket

import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, degree, perturb, out):
    import datetime

    import torch
    import torch.distributed as dist

    from meltpooldg_b200 import _lib as L
    from meltpooldg_b200 import heat as H
    from meltpooldg_b200 import slab as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        cells = (4, 3, 7)
        mesh = H.box_mesh(degree, cells, (0, 0, 0), (1.0, 0.9, 1.6), perturb, 3)
        mat = H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5)
        A = S.SlabHeatOperator(mesh, S.SlabExchange())
        G = H.HeatDiffuseOperator(mesh)
        for op in (A, G):
            op.set_material(mat)
            op.reset_time_increment(1e-2)
        g = torch.Generator(device="cuda").manual_seed(9)
        N = G.n_dofs
        src = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
        T = G.distribute_constraints(torch.rand(N, dtype=torch.float64, device="cuda",
                                                generator=g))
        To = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
        q = 5 * torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
        Tl, Tol = A.local_part(T), A.local_part(To)
        A.set_linearization(Tl, Tol)
        G.set_linearization(T, To)

        def rel(a, b):
            return ((a - b).abs().max() / b.abs().max()).item()
        res = {}
        res["vmult"] = rel(A.vmult(A.new_vector(), A.local_part(src)),
                           A.local_part(G.vmult(G.new_vector(), src)))
        res["diag"] = rel(A.compute_inverse_diagonal(A.new_vector()),
                          A.local_part(G.compute_inverse_diagonal_from_matrixfree(G.new_vector())))
        res["rhs"] = rel(A.create_rhs(A.new_vector(), Tol, A.local_part(q)),
                         A.local_part(G.create_rhs(G.new_vector(), To, q)))
        res["l2"] = abs(A.l2_norm(Tl) - G.l2_norm(T)) / G.l2_norm(T)
        # two implicit Newton steps: slabs (Jacobi-CG) vs the whole mesh's device step
        lin = H.LinearSolverData(rel_tolerance=1e-12, abs_tolerance=0.0)
        nl = H.NonlinearSolverData(residual_tolerance=1e-9)
        op_s = S.SlabHeatOperation(A, lin, nl)
        op_s.set_initial_condition(Tl)
        op_s.heat_source = A.local_part(q)
        op_g = H.HeatDiffuseOperation(G, lin, nl)
        op_g.set_initial_condition(T)
        op_g.heat_source = q
        for _ in range(2):
            op_s.solve(1e-2)
            op_g.solve(1e-2)
        res["steps"] = rel(op_s.T, A.local_part(op_g.T))
        res["newton"] = op_s.newton_iterations
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("degree,perturb", [(2, 0.0), (3, 0.15)])
def test_cuda_slabs_reproduce_the_whole_mesh(degree, perturb):
    world = 2
    with mp.get_context("spawn").Manager() as m:  # no fork of this process
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), degree, perturb, out),
                           nprocs=world, join=True, start_method="spawn")
        out = dict(out)
    assert sorted(out) == [0, 1]
    for r, res in out.items():
        assert res["vmult"] <= 1e-12 and res["diag"] <= 1e-12 and res["rhs"] <= 1e-12, (r, res)
        assert res["l2"] <= 1e-12, (r, res)
        assert res["steps"] <= 1e-8 and res["newton"] >= 1, (r, res)


def test_slab_handle_rejects_bad_ranges():
    from meltpooldg_b200 import heat as H
    mesh = H.box_mesh(2, (3, 3, 4))
    for z in [(-1, 2), (2, 2), (1, 5)]:
        with pytest.raises(H.ExcInvalidArgument):
            H.HeatDiffuseOperator(mesh, slab=z)
    a = H.HeatDiffuseOperator(mesh, slab=(1, 3))
    assert a.n_dofs == 7 * 7 * 5 and a.dims == (7, 7, 5)
