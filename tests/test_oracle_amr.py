"""The two-level (hanging-node) restatement of the heat operator, oracle/amr.py, against the
structured oracle where the two meshes coincide, and against solutions the constrained FE space
holds exactly where they do not."""
import numpy as np
import pytest

from oracle import amr as A
from oracle import oracle as O


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("case", ["unrefined", "refined"])
def test_matches_structured_oracle_without_hanging_nodes(p, case):
    """No cell refined, or every cell refined: the same operator as the structured oracle on
    the coarse or the twice finer box (constant law and the linear-k tangent)."""
    if case == "unrefined":
        mesh = A.TwoLevelBoxMesh(p, (3, 2, 2))
        o = O.Oracle(p, (3, 2, 2))
    else:
        mesh = A.TwoLevelBoxMesh(p, (2, 2, 1), refine=np.ones((1, 2, 2), dtype=bool))
        o = O.Oracle(p, (4, 4, 2))
    assert not mesh.hanging.any()
    assert mesh.n_dofs == o.n_dofs
    assert np.abs(mesh.support_points() - o.support_points()).max() < 1e-13
    assert np.array_equal(mesh.mask, o.mask().astype(bool))
    rng = np.random.default_rng(10 + p)
    src = rng.uniform(-1.0, 1.0, mesh.n_dofs)
    dt = 1e-2
    o.set_material(O.material(O.LAW_CONSTANT, rho=2.0, cp=1.5, k=0.7), dt)
    assert _rel(mesh.vmult(src, rho_cp=3.0, dt=dt, k0=0.7), o.vmult(src)) < 1e-12
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), dt)
    T = o.distribute(rng.uniform(0.0, 1.0, mesh.n_dofs))
    ref = o.vmult(src, T_lin=T)
    assert _rel(mesh.vmult(src, dt=dt, k0=1.0, k1=0.5, T_lin=T), ref) < 1e-12


REFINE = [(1, 1, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2), (0, 0, 0)]  # a block, a corner cell


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_hanging_constraints_interpolate_the_coarse_space(p):
    """Every hanging node's weights sum to one and reproduce any global Q_p function."""
    mesh = A.TwoLevelBoxMesh(p, (4, 3, 3), refine=REFINE)
    assert mesh.hanging.any()
    rows = mesh.C[np.flatnonzero(mesh.hanging)]
    assert np.abs(np.asarray(rows.sum(axis=1)).ravel() - 1.0).max() < 1e-13
    rng = np.random.default_rng(p)
    c = rng.uniform(-1.0, 1.0, (p + 1, p + 1, p + 1))

    def f(x):
        P = [np.stack([x[:, d] ** e for e in range(p + 1)], axis=1) for d in range(3)]
        return np.einsum("ijk,ni,nj,nk->n", c, P[0], P[1], P[2])

    nodes = mesh.lo + mesh.node_pos * mesh.h
    u = f(mesh.support_points())
    assert np.abs(mesh.node_values(u) - f(nodes)).max() < 1e-12 * np.abs(f(nodes)).max()


S = 64.0  # u = S x(1-x) y(1-y) z(1-z) peaks at 1


def _u(x):
    return S * np.prod(x * (1.0 - x), axis=1)


def _grad_u(x):
    q = x * (1.0 - x)
    return S * np.stack([(1.0 - 2.0 * x[:, d]) * np.prod(np.delete(q, d, axis=1), axis=1)
                         for d in range(3)], axis=1)


def _lap_u(x):
    q = x * (1.0 - x)
    return -2.0 * S * sum(np.prod(np.delete(q, d, axis=1), axis=1) for d in range(3))


# (p, tangent): QGauss(p+1) integrates the constant-law forms exactly for p >= 2 and the
# tangent's (k0 + 2 k1 u) grad(u).grad(v) for p >= 3
@pytest.mark.parametrize("p,tangent", [(2, False), (3, False), (4, False), (3, True), (4, True)])
def test_galerkin_solution_is_exact_for_representable_fields(p, tangent):
    """u = 64 x(1-x) y(1-y) z(1-z) lies in the constrained space for p >= 2: the heat
    operator's Galerkin solution with the matching load reproduces it at every DoF, and the
    same mesh with its hanging nodes left free (a planted mistake) does not."""
    refine = [(1, 1, 1), (2, 1, 1), (0, 2, 2)]
    rho_cp, dt, k0, k1 = 2.0, 0.1, 1.0, (0.5 if tangent else 0.0)

    def load(x):
        # strong form of rho_cp/dt w - div((k0 + k1 T) grad(w) + k1 grad(T) w) at T = w = u
        val = rho_cp / dt * _u(x)
        if tangent:
            return (val - (k0 + 2.0 * k1 * _u(x)) * _lap_u(x)
                    - 2.0 * k1 * (_grad_u(x) ** 2).sum(axis=1))
        return val - k0 * _lap_u(x)

    errs = []
    for constrained in (True, False):
        mesh = A.TwoLevelBoxMesh(p, (3, 3, 3), refine=refine, constrain_hanging=constrained)
        assert mesh.hanging.any() == constrained
        T = _u(mesh.support_points())
        x = mesh.solve(mesh.load_vector(load), rho_cp=rho_cp, dt=dt, k0=k0, k1=k1,
                       T_lin=T if tangent else None)
        exact = np.where(mesh.mask, 0.0, T)
        errs.append(np.abs(x - exact).max() / np.abs(exact).max())
    assert errs[0] < 1e-10
    assert errs[1] > 1e-6


def test_constrained_operator_is_symmetric_positive_definite():
    mesh = A.TwoLevelBoxMesh(3, (3, 3, 2), refine=[(1, 1, 0), (0, 0, 1)])
    Amat = mesh.assemble(rho_cp=1.0, dt=1e-3, k0=2.0)
    free = np.flatnonzero(~mesh.mask)
    Af = Amat[free][:, free].toarray()
    assert np.abs(Af - Af.T).max() < 1e-12 * np.abs(Af).max()
    assert np.linalg.eigvalsh(Af).min() > 0.0
    # the mass part integrates the constant function to the volume
    M = mesh.assemble(rho_cp=1.0, dt=1.0, k0=0.0)
    one = np.ones(mesh.n_dofs)
    assert abs(one @ (M @ one) - 1.0) < 1e-12


@pytest.mark.parametrize("p", [1, 2, 3])
def test_cellwise_constraints_match_the_condensed_operator(p):
    """The second form: each refined cell gathers its coarse neighbours' face and edge DoFs and
    interpolates them with the 1D child matrices, one direction at a time (the cell kernel's
    form); cell by cell it gives the constrained nodal values, and its operator equals
    C^T A C. The refinement has cells with hanging faces, with two hanging faces and with
    hanging edges only (the coarse cell (2, 2, 1) touches (1, 1, 1)'s children on one edge)."""
    mesh = A.TwoLevelBoxMesh(p, (4, 3, 3), refine=REFINE)
    codes = [mesh.hanging_code(c) for c in range(mesh.n_cells)]
    assert any(c & 0o70 for c in codes) and any(c & 0o700 for c in codes)
    assert any(bin(c & 0o70).count("1") >= 2 for c in codes)
    rng = np.random.default_rng(20 + p)
    u = rng.uniform(-1.0, 1.0, mesh.n_dofs)
    nodal = mesh.node_values(u)
    for c in range(mesh.n_cells):
        idx, F = mesh.cell_map(c)
        local = u[idx] if F is None else F @ u[idx]
        assert np.abs(local - nodal[mesh.cell_nodes[c]]).max() < 1e-13
    coef = dict(rho_cp=2.0, dt=0.05, k0=1.0)
    assert _rel(mesh.vmult_cellwise(u, **coef), mesh.vmult(u, **coef)) < 1e-13
    T = np.where(mesh.mask, 0.0, rng.uniform(0.0, 1.0, mesh.n_dofs))
    coef = dict(rho_cp=1.0, dt=0.05, k0=1.0, k1=0.5, T_lin=T)
    assert _rel(mesh.vmult_cellwise(u, **coef), mesh.vmult(u, **coef)) < 1e-13


def test_rhs_and_newton_step_match_structured_oracle_without_hanging_nodes():
    """create_rhs and two implicit k(T) = 1 + 0.5 T steps with a Gaussian source: the refined
    mesh with every cell refined against the structured oracle on the twice finer box."""
    p, dt = 2, 1e-2
    mesh = A.TwoLevelBoxMesh(p, (2, 2, 2), refine=np.ones((2, 2, 2), dtype=bool))
    o = O.Oracle(p, (4, 4, 4))
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), dt)
    rng = np.random.default_rng(3)
    T = o.distribute(rng.uniform(0.0, 1.0, o.n_dofs))
    To = rng.uniform(0.0, 1.0, o.n_dofs)
    q = o.gaussian_source(50.0, (0.5, 0.5, 0.9), 0.2)
    ref = o.create_rhs(T, To, q)
    got = mesh.create_rhs(T, To, q, dt=dt, k0=1.0, k1=0.5)
    assert _rel(got, ref) < 1e-12
    Ta, Toa = T.copy(), T.copy()
    Tb, Tob = T.copy(), T.copy()
    for _ in range(2):
        rc, _ = o.time_step_newton(Ta, Toa, dt, dt, q, res_tol=1e-9, corr_tol=1e-10,
                                   solver="cg")
        assert rc == 0
        mesh.time_step_newton(Tb, Tob, dt, dt, q, k0=1.0, k1=0.5)
    assert _rel(Tb, Ta) < 1e-9
    assert _rel(Tob, Toa) < 1e-9


def test_newton_step_with_hanging_nodes_converges_to_the_residual_tolerance():
    mesh = A.TwoLevelBoxMesh(2, (3, 3, 3), refine=[(1, 1, 1), (2, 1, 1), (1, 2, 2)])
    x = mesh.support_points()
    q = 50.0 * np.exp(-((x - np.array([0.5, 0.5, 0.6])) ** 2).sum(axis=1) / 0.2 ** 2)
    T = np.where(mesh.mask, 0.0, 0.5 * _u(x))
    To = T.copy()
    its = mesh.time_step_newton(T, To, 1e-2, 1e-2, q, k0=1.0, k1=0.5)
    assert 1 < its <= 5
    r = mesh.create_rhs(T, To, q, dt=1e-2, k0=1.0, k1=0.5)
    assert np.linalg.norm(r) < 1e-9


@pytest.mark.parametrize("p", [1, 2, 3])
def test_cellwise_diagonal_and_residual_match_the_condensed_forms(p):
    """The inverse diagonal (the reference's |d| > 1e-10 rule) and create_rhs accumulated cell
    by cell with the in-cell constraints equal those of C^T A C, with hanging faces and edges."""
    mesh = A.TwoLevelBoxMesh(p, (4, 3, 3), refine=REFINE)
    rng = np.random.default_rng(40 + p)
    T = rng.uniform(0.0, 1.0, mesh.n_dofs)
    To = rng.uniform(0.0, 1.0, mesh.n_dofs)
    q = rng.uniform(0.0, 5.0, mesh.n_dofs)
    for coef in (dict(rho_cp=2.0, dt=0.05, k0=1.0),
                 dict(rho_cp=1.0, dt=0.05, k0=1.0, k1=0.5, T_lin=T)):
        a = mesh.inverse_diagonal(**coef)
        b = mesh.inverse_diagonal_cellwise(**coef)
        assert _rel(b, a) < 1e-13
        assert np.all(a[mesh.mask] == 1.0)
    kw = dict(rho_cp=2.0, dt=0.05, k0=1.0, k1=0.5)
    a = mesh.create_rhs(T, To, q, **kw)
    b = mesh.create_rhs_cellwise(T, To, q, **kw)
    assert _rel(b, a) < 1e-13
    assert np.all(b[mesh.mask] == 0.0)


def _three_levels():
    lev = np.zeros((5, 5, 5), dtype=np.int64)
    lev[1:4, 1:4, 1:4] = 1
    lev[2, 2, 2] = 2
    return lev


def test_multilevel_mesh_reduces_to_the_two_level_and_structured_meshes():
    rng = np.random.default_rng(50)
    lev = np.zeros((3, 3, 4), dtype=np.int64)
    for ix, iy, iz in REFINE:
        lev[iz, iy, ix] = 1
    a = A.MultiLevelBoxMesh(2, (4, 3, 3), lev)
    b = A.TwoLevelBoxMesh(2, (4, 3, 3), refine=REFINE)
    assert a.n_dofs == b.n_dofs and a.hanging.sum() == b.hanging.sum()
    assert np.abs(a.support_points() - b.support_points()).max() < 1e-14
    u = rng.uniform(-1.0, 1.0, a.n_dofs)
    assert np.abs(a.node_values(u) - b.node_values(u)).max() < 1e-14
    coef = dict(rho_cp=2.0, dt=0.05, k0=1.0)
    assert _rel(a.vmult(u, **coef), b.vmult(u, **coef)) < 1e-13
    assert [a.hanging_code(c) for c in range(a.n_cells)] == \
        [b.hanging_code(c) for c in range(b.n_cells)]
    # every cell twice refined: the structured oracle on the four times finer box
    c = A.MultiLevelBoxMesh(2, (2, 1, 1), np.full((1, 1, 2), 2))
    o = O.Oracle(2, (8, 4, 4))
    o.set_material(O.material(O.LAW_CONSTANT, rho=2.0, cp=1.0, k=1.0), 0.05)
    v = rng.uniform(-1.0, 1.0, c.n_dofs)
    assert c.n_dofs == o.n_dofs and not c.hanging.any()
    assert _rel(c.vmult(v, **coef), o.vmult(v)) < 1e-12


def test_unbalanced_levels_are_rejected():
    lev = np.zeros((1, 1, 2), dtype=np.int64)
    lev[0, 0, 1] = 2
    with pytest.raises(ValueError):
        A.MultiLevelBoxMesh(2, (2, 1, 1), lev)


@pytest.mark.parametrize("p", [2, 3])
def test_three_level_mesh_constraints_and_galerkin_exactness(p):
    """Levels 0, 1 and 2 (2:1 balanced): constraint weights reproduce Q_p, the cell-wise form
    equals C^T A C, and the Galerkin solution reproduces u = 64 x(1-x) y(1-y) z(1-z)."""
    mesh = A.MultiLevelBoxMesh(p, (5, 5, 5), _three_levels())
    lv = mesh.cell_level
    assert set(np.unique(lv)) == {0, 1, 2}
    codes = [mesh.hanging_code(c) for c in range(mesh.n_cells)]
    assert any(codes[c] for c in np.flatnonzero(lv == 2))  # level-2 cells hang on level 1
    rng = np.random.default_rng(60 + p)
    u = rng.uniform(-1.0, 1.0, mesh.n_dofs)
    nodal = mesh.node_values(u)
    for c in range(mesh.n_cells):
        idx, F = mesh.cell_map(c)
        local = u[idx] if F is None else F @ u[idx]
        assert np.abs(local - nodal[mesh.cell_nodes[c]]).max() < 1e-13
    coef = dict(rho_cp=2.0, dt=0.1, k0=1.0)
    assert _rel(mesh.vmult_cellwise(u, **coef), mesh.vmult(u, **coef)) < 1e-13

    def load(x):
        return 2.0 / 0.1 * _u(x) - _lap_u(x)

    x = mesh.solve(mesh.load_vector(load), **coef)
    exact = np.where(mesh.mask, 0.0, _u(mesh.support_points()))
    assert np.abs(x - exact).max() < 1e-10 * np.abs(exact).max()
