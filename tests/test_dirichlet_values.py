"""Dirichlet values that change between steps (HeatData::enable_time_dependent_bc): the oracle's
setter against values given at creation, the first-face rule at edges, and the product's
argument checks without a GPU."""
import ctypes

import numpy as np

from meltpooldg_b200 import _lib as L
from oracle import oracle as O

VALS = (1.0, 2.0, 3.0, 4.0, 5.0, 6.0)


def test_values_set_later_equal_values_given_at_creation():
    a = O.Oracle(2, (3, 3, 3), dirichlet_value=VALS)
    b = O.Oracle(2, (3, 3, 3))
    b.set_dirichlet_values(VALS)
    rng = np.random.default_rng(1)
    u = rng.uniform(0.0, 1.0, a.n_dofs)
    assert np.array_equal(a.distribute(u.copy()), b.distribute(u.copy()))
    for o in (a, b):
        o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), 1e-2)
    T0 = rng.uniform(0.0, 1.0, a.n_dofs)
    Ta, Toa, Tb, Tob = T0.copy(), T0.copy(), T0.copy(), T0.copy()
    assert a.time_step_newton(Ta, Toa, 1e-2, 1e-2, solver="cg")[0] == 0
    assert b.time_step_newton(Tb, Tob, 1e-2, 1e-2, solver="cg")[0] == 0
    assert np.abs(Ta - Tb).max() <= 1e-12 * np.abs(Ta).max()  # threaded reductions


def test_first_flagged_face_owns_edges_and_a_step_takes_new_values():
    o = O.Oracle(1, (2, 2, 2))
    o.set_material(O.material(), 1e-2)
    o.set_dirichlet_values(VALS)
    x = o.support_points()
    u = o.distribute(np.zeros(o.n_dofs))
    on = lambda d, v: np.abs(x[:, d] - v) < 1e-12
    assert np.all(u[on(0, 0.0)] == 1.0)                     # x- owns its edges and corners
    assert np.all(u[on(1, 1.0) & ~on(0, 0.0) & ~on(0, 1.0)] == 4.0)
    assert np.all(u[on(2, 1.0) & ~on(0, 0.0) & ~on(0, 1.0) & ~on(1, 0.0) & ~on(1, 1.0)] == 6.0)
    T, To = u.copy(), u.copy()
    new = tuple(v + 10.0 for v in VALS)
    o.set_dirichlet_values(new)
    assert o.time_step_newton(T, To, 1e-2, 1e-2, solver="cg")[0] == 0
    m = o.mask().astype(bool)
    assert np.all(T[m] == o.distribute(np.zeros(o.n_dofs))[m])
    assert np.all(T[on(0, 0.0)] == 11.0)


def test_product_setter_rejects_missing_arguments_without_gpu():
    lib = L.load()
    v = (ctypes.c_double * 6)(*VALS)
    assert lib.mpdg_heat_set_dirichlet_values(None, v) == L.ERR_INVALID_ARGUMENT
