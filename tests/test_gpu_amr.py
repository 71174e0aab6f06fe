"""The hanging-node cell kernel (mpdg_amr_vmult) against the oracle's two-level operator, and
against the structured GPU operator where no cell is refined."""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from meltpooldg_b200.amr import AmrHeatOperator
from oracle import amr as A

pytestmark = pytest.mark.gpu

# cells with one, two and three hanging faces, a face and an edge, and hanging edges only
REFINE = [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2), (0, 0, 0)]
BOX = dict(hi=(2.0, 1.5, 1.0), dirichlet=("x-", "y+", "z-", "z+"))


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("law", ["constant", "linear_k"])
def test_vmult_with_hanging_nodes_matches_oracle(p, law):
    cells = (4, 3, 3)
    op = AmrHeatOperator(H.box_mesh(p, cells, **BOX), REFINE, device=0)
    o = A.TwoLevelBoxMesh(p, cells, refine=REFINE, **BOX)
    assert op.n_dofs == o.n_dofs and o.hanging.any()
    rng = np.random.default_rng(30 + p)
    src = rng.uniform(-1.0, 1.0, o.n_dofs)
    dt = 1e-2
    if law == "constant":
        op.set_material(H.material(rho=2.0, cp=1.5, k=0.7), dt)
        ref = o.vmult(src, rho_cp=3.0, dt=dt, k0=0.7)
        T = None
    else:
        op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5), dt)
        Tn = rng.uniform(0.0, 1.0, o.n_dofs)
        ref = o.vmult(src, rho_cp=1.0, dt=dt, k0=1.0, k1=0.5, T_lin=Tn)
        T = torch.tensor(Tn, device="cuda")
    dst = torch.empty(o.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, torch.tensor(src, device="cuda"), T)
    got = dst.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_unrefined_mesh_matches_structured_operator():
    p, cells = 3, (5, 4, 3)
    mesh = H.box_mesh(p, cells, **BOX)
    amr = AmrHeatOperator(mesh, (), device=0)
    st = H.HeatDiffuseOperator(mesh)
    assert amr.n_dofs == st.n_dofs
    dt = 5e-3
    m = H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5)
    amr.set_material(m, dt)
    st.set_material(m)
    st.reset_time_increment(dt)
    g = torch.Generator(device="cuda").manual_seed(4)
    T = torch.rand(st.n_dofs, dtype=torch.float64, device="cuda", generator=g)
    src = torch.rand(st.n_dofs, dtype=torch.float64, device="cuda", generator=g)
    st.set_linearization(T, T)
    a = torch.empty_like(src)
    b = torch.empty_like(src)
    amr.vmult(a, src, T)
    st.vmult(b, src)
    assert (a - b).abs().max().item() <= 1e-12 * b.abs().max().item()


def _coef(law):
    if law == "constant":
        return H.material(rho=2.0, cp=1.5, k=0.7), dict(rho_cp=3.0, k0=0.7)
    return H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5), dict(rho_cp=1.0, k0=1.0, k1=0.5)


def cuda(a):
    return torch.tensor(a, dtype=torch.float64, device="cuda")


def _relmax(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else a
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("law", ["constant", "linear_k"])
def test_diagonal_and_residual_with_hanging_nodes_match_oracle(p, law):
    cells = (4, 3, 3)
    op = AmrHeatOperator(H.box_mesh(p, cells, **BOX), REFINE, device=0)
    o = A.TwoLevelBoxMesh(p, cells, refine=REFINE, **BOX)
    m, coef = _coef(law)
    dt = 1e-2
    op.set_material(m, dt)
    rng = np.random.default_rng(40 + p)
    N = o.n_dofs
    T, To, q = rng.uniform(0, 1, N), rng.uniform(0, 1, N), rng.uniform(0, 3, N)
    lin = dict(T_lin=T) if law == "linear_k" else {}
    ref = o.inverse_diagonal(dt=dt, **coef, **lin)
    got = op.inverse_diagonal(torch.empty(N, dtype=torch.float64, device="cuda"),
                              cuda(T) if law == "linear_k" else None)
    assert _relmax(1.0 / got.cpu().numpy(), 1.0 / ref) <= 1e-12
    base = rng.uniform(-1, 1, N)
    rref = o.create_rhs(T, To, q, dst=base.copy(), dt=dt,
                        **{k: v for k, v in coef.items() if k != "T_lin"})
    d = cuda(base)
    op.create_rhs(d, cuda(T), cuda(To), cuda(q))
    assert _relmax(d, rref) <= 1e-12


MULTI = np.zeros((5, 5, 5), dtype=np.uint8)
MULTI[1:4, 1:4, 1:4] = 1
MULTI[2, 2, 2] = 2  # levels 0, 1 and 2 under the 2:1 balance


@pytest.mark.parametrize("p", [2, 3])
def test_multilevel_operator_matches_oracle(p):
    cells = (5, 5, 5)
    op = AmrHeatOperator(H.box_mesh(p, cells, **BOX), MULTI, device=0)
    o = A.MultiLevelBoxMesh(p, cells, MULTI, **BOX)
    assert op.n_dofs == o.n_dofs and o.hanging.any()
    m, coef = _coef("linear_k")
    op.set_material(m, 1e-2)
    rng = np.random.default_rng(5)
    src, T = rng.uniform(-1, 1, o.n_dofs), rng.uniform(0, 1, o.n_dofs)
    ref = o.vmult(src, dt=1e-2, T_lin=T, **coef)
    dst = torch.empty(o.n_dofs, dtype=torch.float64, device="cuda")
    op.vmult(dst, cuda(src), cuda(T))
    assert _relmax(dst, ref) <= 1e-12
    dref = o.inverse_diagonal(dt=1e-2, T_lin=T, **coef)
    got = op.inverse_diagonal(torch.empty_like(dst), cuda(T))
    assert _relmax(1.0 / got.cpu().numpy(), 1.0 / dref) <= 1e-12


def test_linear_solve_with_hanging_nodes_matches_direct_solve():
    p, cells = 2, (4, 3, 3)
    op = AmrHeatOperator(H.box_mesh(p, cells, **BOX), REFINE, device=0)
    o = A.TwoLevelBoxMesh(p, cells, refine=REFINE, **BOX)
    m, coef = _coef("linear_k")
    op.set_material(m, 1e-2)
    rng = np.random.default_rng(8)
    T = rng.uniform(0, 1, o.n_dofs)
    b = o.vmult(rng.uniform(-1, 1, o.n_dofs), dt=1e-2, T_lin=T, **coef)
    x_ref = o.solve(b, dt=1e-2, T_lin=T, **coef)
    x = torch.zeros(o.n_dofs, dtype=torch.float64, device="cuda")
    its = op.linear_solve(x, cuda(b), cuda(T), rel_tolerance=1e-13)
    assert its > 0
    assert _relmax(x, x_ref) <= 1e-10


@pytest.mark.parametrize("mesh", ["two_level", "multilevel"])
def test_implicit_steps_on_refined_mesh_match_oracle(mesh):
    """Three implicit k(T) steps (linear predictor, history commit, Newton with Jacobi-CG
    increment solves) against the oracle's Newton step with exact solves, to 1e-9."""
    p, dt = 2, 1e-2
    if mesh == "two_level":
        cells, ref_arg = (4, 3, 3), REFINE
        o = A.TwoLevelBoxMesh(p, cells, refine=REFINE, **BOX)
    else:
        cells, ref_arg = (5, 5, 5), MULTI
        o = A.MultiLevelBoxMesh(p, cells, MULTI, **BOX)
    op = AmrHeatOperator(H.box_mesh(p, cells, **BOX), ref_arg, device=0)
    m, coef = _coef("linear_k")
    op.set_material(m, dt)
    x = o.support_points()
    T0 = np.where(o.mask, 0.0, np.sin(np.pi * x[:, 0] / 2.0) * (1.0 + x[:, 2]))
    q = 5.0 * np.exp(-((x[:, 0] - 1.0) ** 2 + (x[:, 1] - 0.7) ** 2) / 0.2)
    T, To = T0.copy(), T0.copy()
    Tg, Tog = cuda(T0), cuda(T0)
    prm = H.step_params(H.LinearSolverData(rel_tolerance=1e-13),
                        H.NonlinearSolverData(residual_tolerance=1e-9))
    dt_old = 0.0
    for step in range(3):
        o.time_step_newton(T, To, dt, dt_old, heat_source=q, **coef)
        st = op.time_step(Tg, Tog, dt, dt_old, cuda(q), prm)
        assert st.converged == 1 and st.newton_iterations >= 2
        dt_old = dt
        assert _relmax(Tg, T) <= 1e-9, step
        assert _relmax(Tog, To) <= 1e-9, step
