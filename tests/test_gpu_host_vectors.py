"""The OperatorMatrixFree verbs on HOST vectors through the C ABI (mpdg_heat_*_host), the entry
points a MeltPoolDG adapter binds: its VectorType is the host
LinearAlgebra::distributed::Vector<double> (operator_base.hpp:192) in deal.II's DoF numbering.

Checked against the oracle at 1e-12 relative, with the identity numbering and with a seeded
random DoF permutation (the caller's numbering), and a host-side Jacobi-CG that calls only the
host verbs (what LinearSolver::solve does with such an operator, linear_solver.hpp:22-134)
reproduces the oracle's CG solution."""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def pair(degree=3, cells=(5, 4, 6), perturb=0.2, dt=1e-3):
    o = O.Oracle(degree, cells, perturb=perturb, seed=12)
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), dt)
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, perturb=perturb, seed=12))
    g.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
    g.reset_time_increment(dt)
    return o, g


@pytest.mark.parametrize("permuted", [False, True])
def test_host_verbs_match_oracle(permuted):
    o, g = pair()
    N = o.n_dofs
    rng = np.random.default_rng(4)
    # lex[i]: lexicographic index of the caller's DoF i
    lex = rng.permutation(N).astype(np.int64) if permuted else np.arange(N, dtype=np.int64)
    g.set_dof_permutation(lex)
    to_caller = lambda v: v[lex]  # caller vector c with c[i] = v[lex[i]]
    src, Tl, To, q = (rng.uniform(-1, 1, N), o.distribute(rng.uniform(0, 1, N)),
                      rng.uniform(0, 1, N), rng.uniform(0, 5, N))
    g.set_linearization_host(to_caller(Tl), to_caller(To))
    dst = g.vmult_host(np.empty(N), to_caller(src))
    assert rel(dst, to_caller(o.vmult(src, Tl, To))) <= TOL64
    d = g.compute_inverse_diagonal_host(np.empty(N))
    assert rel(1.0 / d, to_caller(1.0 / o.inverse_diagonal(Tl, To))) <= TOL64
    base = rng.uniform(-1, 1, N)
    r = g.create_rhs_host(to_caller(base), to_caller(To), to_caller(q))
    assert rel(r, to_caller(o.create_rhs(Tl, To, q, dst=base.copy()))) <= TOL64
    # the device verbs keep the lexicographic numbering
    y = g.vmult(g.new_vector(), torch.tensor(src, device="cuda"))
    assert rel(y.cpu().numpy(), o.vmult(src, Tl, To)) <= TOL64


def test_host_jacobi_cg_matches_oracle():
    """deal.II SolverCG semantics on the host, every operator application through the host
    verbs in a permuted numbering: the solution equals the oracle's to the solver tolerance."""
    o, g = pair(degree=2, cells=(6, 5, 4), perturb=0.1)
    N = o.n_dofs
    rng = np.random.default_rng(8)
    lex = rng.permutation(N).astype(np.int64)
    g.set_dof_permutation(lex)
    Tl = o.distribute(rng.uniform(0, 1, N))
    g.set_linearization_host(Tl[lex], Tl[lex])
    b = o.vmult(rng.uniform(-1, 1, N), Tl, Tl)
    x_ref, its_ref, _ = o.cg(b, T_lin=Tl, T_old=Tl, rel_tol=1e-12)
    inv_d = g.compute_inverse_diagonal_host(np.empty(N))
    bb = b[lex]
    x = np.zeros(N)
    r = bb.copy()
    z = inv_d * r
    p = z.copy()
    rz = r @ z
    r0 = np.linalg.norm(r)
    its = 0
    Ap = np.empty(N)
    while np.linalg.norm(r) > 1e-12 * r0 and its < 1000:
        g.vmult_host(Ap, p)
        alpha = rz / (p @ Ap)
        x += alpha * p
        r -= alpha * Ap
        z = inv_d * r
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
        its += 1
    assert abs(its - its_ref) <= 2
    x_lex = np.empty(N)
    x_lex[lex] = x
    assert rel(x_lex, x_ref) <= 1e-9


def test_invalid_permutation_and_host_arguments_are_rejected():
    _, g = pair(degree=1, cells=(2, 2, 2), perturb=0.0)
    N = g.n_dofs
    bad = np.arange(N, dtype=np.int64)
    bad[3] = bad[4]  # repeated entry
    with pytest.raises(H.ExcInvalidArgument):
        g.set_dof_permutation(bad)
    bad = np.arange(N, dtype=np.int64)
    bad[0] = N  # out of range
    with pytest.raises(H.ExcInvalidArgument):
        g.set_dof_permutation(bad)
    with pytest.raises(H.ExcInvalidArgument):
        g.vmult_host(np.empty(N - 1), np.empty(N))
    with pytest.raises(H.ExcInvalidArgument):
        g.vmult_host(np.empty(N), torch.zeros(N, dtype=torch.float64, device="cuda"))
    g.set_dof_permutation(None)  # identity again
    T = np.zeros(N)
    g.set_linearization_host(T, T)
    x = np.ones(N)
    assert np.isfinite(g.vmult_host(np.empty(N), x)).all()
