"""The FP32 Picard operator of the multigrid fine level on the tensor cores (k_vmult_picard_tc:
tcgen05 TF32 GEMMs over bricks of 8 x 4 x 4 cells, FE_Q(3), uniform box meshes; opt-in) against
the oracle's Picard form, against the CUDA-core FP32 kernel, and inside the preconditioned solve.

Meshes with partial bricks in every direction, a single cell, anisotropic cells, Dirichlet faces
(all, two, none) and Robin faces. Tolerance: 5e-3 relative in the max norm (TF32 operands carry
10 mantissa bits; the CUDA-core FP32 kernel is held to 2e-5 by the other parity tests)."""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_TF32 = 5e-3
DT = 5e-4


def cuda(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def rel(a, b):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().double().numpy()
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def pair(cells, dirichlet=0x3F, hi=(1.0, 1.0, 1.0), degree=3, perturb=0.0):
    o = O.Oracle(degree, cells, hi=hi, perturb=perturb, seed=3, dirichlet_mask=dirichlet)
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), DT)
    faces = [f for f in range(6) if dirichlet & (1 << f)]
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, (0.0, 0.0, 0.0), hi, perturb, 3, faces,
                                         [0.0] * 6))
    g.set_material(H.material(law=L.LAW_LINEAR_K, rho=1.0, cp=1.0, k=1.0, k1=0.5))
    g.reset_time_increment(DT)
    return o, g


@pytest.mark.parametrize("cells", [(8, 4, 4), (9, 5, 6), (17, 3, 9), (1, 1, 1), (2, 7, 5)])
@pytest.mark.parametrize("dirichlet", [0x3F, 0b110000, 0])
def test_tensor_core_picard_operator_matches_oracle(cells, dirichlet):
    hi = (1.0, 0.6, 1.3) if cells[0] % 2 else (1.0, 1.0, 1.0)
    o, g = pair(cells, dirichlet, hi)
    if dirichlet != 0x3F:  # Robin terms on a free face (added before the cell kernel)
        o.set_boundary(0, convection=(5.0, 300.0))
        g.set_boundary(0, convection=(5.0, 300.0))
    assert not g.picard_tensor_cores  # opt-in
    g.set_picard_tensor_cores(True)
    assert g.picard_tensor_cores
    rng = np.random.default_rng(sum(cells) + dirichlet)
    N = o.n_dofs
    src, Tl = rng.uniform(-1, 1, N), rng.uniform(0.0, 2.0, N)
    g.set_linearization(cuda(Tl), cuda(Tl))
    ref = o.vmult(src, Tl, Tl, form=2)
    y = g.vmult_picard_f32(g.new_vector(torch.float32), cuda(src, torch.float32))
    e = rel(y, ref)
    print(f"{cells} mask {dirichlet:#x}: rel max error {e:.2e}")
    assert e <= TOL_TF32
    # constrained rows stay zero
    cons = o.mask().astype(bool)
    assert cons.any() == bool(dirichlet)
    assert np.all(y.cpu().numpy()[cons] == 0.0)


def test_tensor_core_against_cuda_core_kernel_multi_brick():
    """48^3 cells (1,728 bricks, several per CTA): the TF32 kernel against the FP32 one on a
    smooth input (slowly varying: the stiffness part of A u cancels, so the relative error is a
    few TF32 units, measured 2.9e-3) and on a random one (no cancellation)."""
    cells = (48, 48, 48)
    g = H.HeatDiffuseOperator(H.box_mesh(3, cells))
    g.set_material(H.material(law=L.LAW_LINEAR_K, rho=1.0, cp=1.0, k=1.0, k1=0.5))
    g.reset_time_increment(DT)
    N = g.n_dofs
    gen = torch.Generator(device="cuda").manual_seed(1)
    Tl = torch.rand(N, device="cuda", dtype=torch.float64, generator=gen)
    g.set_linearization(Tl, Tl)
    x = torch.linspace(0, 1, N, device="cuda", dtype=torch.float64)
    for src, tol in ((torch.sin(7 * x).float(), 1e-2),
                     (torch.rand(N, device="cuda", generator=gen) - 0.5, 2e-3)):
        g.set_picard_tensor_cores(False)
        ref = g.vmult_picard_f32(g.new_vector(torch.float32), src).double()
        g.set_picard_tensor_cores(True)
        y = g.vmult_picard_f32(g.new_vector(torch.float32), src).double()
        l2 = (torch.linalg.vector_norm(y - ref) / torch.linalg.vector_norm(ref)).item()
        print(f"TF32 vs FP32 kernel: rel L2 {l2:.2e}")
        assert l2 <= tol
        assert rel(y, ref.cpu().numpy()) <= 2 * tol


def test_only_where_the_kernel_exists():
    for degree, perturb in ((2, 0.0), (4, 0.0), (3, 0.2)):
        g = H.HeatDiffuseOperator(H.box_mesh(degree, (4, 4, 4), perturb=perturb))
        g.set_picard_tensor_cores(True)
        assert not g.picard_tensor_cores
    g = H.HeatDiffuseOperator(H.box_mesh(3, (4, 4, 4)))
    assert not g.picard_tensor_cores  # opt-in: the CUDA-core kernel is the default
    g.set_picard_tensor_cores(True)
    assert g.picard_tensor_cores
    g.set_picard_tensor_cores(False)
    assert not g.picard_tensor_cores


def test_multigrid_solve_with_the_tensor_core_fine_level():
    """One implicit k(T) step on 32^3 cells with the benchmark's solver (FP64 flexible CG, FP32
    p-multigrid, Picard operators): the fine level on the tensor cores and on the CUDA cores
    converge to the same tolerance, the fields agree to it, and the outer iteration count grows
    by at most one."""
    cells = (32, 32, 32)
    res = {}
    for tc in (False, True):
        g = H.HeatDiffuseOperator(H.box_mesh(3, cells))
        g.set_material(H.material(law=L.LAW_LINEAR_K, rho=1.0, cp=1.0, k=1.0, k1=0.5))
        g.set_picard_tensor_cores(tc)
        lin = H.LinearSolverData(preconditioner_type=L.PRECOND_MG_F32, rel_tolerance=1e-8,
                                 abs_tolerance=0.0, cheb_picard=True)
        opn = H.HeatDiffuseOperation(g, lin, predictor=L.PREDICTOR_LINEAR,
                                     single_linearization=True)
        q = g.new_vector()
        g.gaussian_source(q, 500.0, (0.4, 0.5, 0.95), 0.05)
        opn.heat_source = q
        its = []
        for _ in range(3):
            st = opn.solve(DT)
            assert st.converged == 1
            its.append(st.linear_iterations)
        res[tc] = (its, opn.T.clone())
    (its0, T0), (its1, T1) = res[False], res[True]
    d = (torch.linalg.vector_norm(T1 - T0) / torch.linalg.vector_norm(T0)).item()
    print(f"outer iterations FP32 fine level {its0}, TF32 {its1}; rel L2 difference {d:.2e}")
    assert d <= 1e-6
    assert all(b <= a + 1 for a, b in zip(its0, its1))
