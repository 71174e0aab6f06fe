"""Time-dependent Dirichlet values on the GPU (HeatData::enable_time_dependent_bc): values set
between steps with mpdg_heat_set_dirichlet_values reach the device distribute and the time step,
with the first flagged face in the order x-, x+, y-, y+, z-, z+ owning edges and corners as in
the oracle; compared with the oracle given the same values, every DoF included."""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu

VALS = (1.0, 2.0, 3.0, 4.0, 5.0, 6.0)


def cuda(a):
    return torch.tensor(a, dtype=torch.float64, device="cuda")


@pytest.mark.parametrize("degree,perturb", [(1, 0.0), (3, 0.2)])
def test_distribute_uses_new_values_on_faces_edges_and_corners(degree, perturb):
    o = O.Oracle(degree, (3, 4, 2), perturb=perturb, seed=6)
    mesh = H.box_mesh(degree, (3, 4, 2), perturb=perturb, seed=6)
    g = H.HeatDiffuseOperator(mesh)
    rng = np.random.default_rng(2)
    u = rng.uniform(-1, 1, o.n_dofs)
    for vals in (VALS, tuple(10.0 * v - 3.0 for v in VALS)):
        o.set_dirichlet_values(vals)
        g.set_dirichlet_values(vals)
        ug = cuda(u)
        g.distribute_constraints(ug)
        assert np.array_equal(ug.cpu().numpy(), o.distribute(u.copy()))
    # the caller's descriptor keeps its values (the operator holds a copy)
    assert tuple(mesh.dirichlet_value) == (0.0,) * 6


def test_partial_dirichlet_faces_and_dict_values():
    mask = 0b101001  # x-, y+, z+
    o = O.Oracle(2, (3, 3, 3), dirichlet_mask=mask)
    g = H.HeatDiffuseOperator(H.box_mesh(2, (3, 3, 3), dirichlet=("x-", "y+", "z+")))
    o.set_dirichlet_values((7.0, 0.0, 0.0, -2.0, 0.0, 0.5))
    g.set_dirichlet_values({"x-": 7.0, "y+": -2.0, "z+": 0.5})
    u = np.random.default_rng(4).uniform(size=o.n_dofs)
    ug = cuda(u)
    g.distribute_constraints(ug)
    assert np.array_equal(ug.cpu().numpy(), o.distribute(u.copy()))


@pytest.mark.parametrize("law", ["constant", "linear_k"])
def test_steps_with_values_changed_between_steps_match_oracle(law):
    """Three Newton steps (linear predictor, CG) with new Dirichlet values before each step."""
    dt = 1e-2
    mat = dict(law=0, k=1.0) if law == "constant" else dict(law=1, k=1.0, k1=0.5)
    o = O.Oracle(2, (4, 3, 3), perturb=0.1, seed=2, dirichlet_value=VALS)
    o.set_material(O.material(**mat), dt)
    g = H.HeatDiffuseOperator(H.box_mesh(2, (4, 3, 3), perturb=0.1, seed=2,
                                         dirichlet_values=dict(zip(H.FACES, VALS))))
    g.set_material(H.material(**mat))
    T0 = o.distribute(np.random.default_rng(1).uniform(0, 1, o.n_dofs))
    T, To = T0.copy(), T0.copy()
    lin = H.LinearSolverData(rel_tolerance=1e-13)
    opn = H.HeatDiffuseOperation(g, lin, H.NonlinearSolverData(residual_tolerance=1e-9))
    opn.set_initial_condition(cuda(T0))
    opn.T_old.copy_(cuda(T0))
    dt_old = 0.0
    for step in range(3):
        vals = tuple(v * (1.0 + 0.5 * (step + 1)) for v in VALS)
        o.set_dirichlet_values(vals)
        g.set_dirichlet_values(vals)
        rc, _ = o.time_step_newton(T, To, dt, dt_old, solver="cg", rel_tol=1e-13)
        assert rc == 0
        st = opn.solve(dt)
        assert st.converged == 1
        dt_old = dt
        err = np.abs(opn.T.cpu().numpy() - T).max() / np.abs(T).max()
        assert err <= 1e-9, (step, err)
        m = o.mask().astype(bool)
        assert np.array_equal(opn.T.cpu().numpy()[m], o.distribute(np.zeros(o.n_dofs))[m])
