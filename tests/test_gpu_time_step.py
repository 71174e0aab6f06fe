"""Implicit heat steps on the GPU: the reference regression case and the
single-linearisation step against the oracle."""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# applications/mp-heat-transfer/cases/unidirectional_heat_transfer/tests/
#   unidirectional_heat_transfer.mpirun=4.output
UNIDIRECTIONAL = [5.64198e-03, 5.53556e-03, 5.44694e-03, 5.37273e-03, 5.31056e-03]


def test_unidirectional_heat_transfer_newton_on_gpu():
    op = H.HeatDiffuseOperator(H.box_mesh(1, (32, 32, 1), (0, 0, 0), (0.1, 0.1, 1.0),
                                          dirichlet=()))
    op.set_material(H.material())
    opn = H.HeatDiffuseOperation(op, H.LinearSolverData(rel_tolerance=1e-12),
                                 H.NonlinearSolverData(residual_tolerance=5e-9))
    x = op.support_points()
    opn.set_initial_condition(x[:, 0].contiguous())
    for ref in UNIDIRECTIONAL:
        st = opn.solve(1e-4)
        assert st.converged == 1
        assert float(f"{op.l2_norm(opn.T):.5e}") == ref


@pytest.mark.parametrize("precond", [L.PRECOND_JACOBI, L.PRECOND_CHEBYSHEV_JACOBI_F32,
                                     L.PRECOND_MG_F32])
def test_single_linearization_step_matches_oracle(precond):
    """One k(T) = 1 + 0.5 T step: T = T_g + J(T_g)^-1 (-R(T_g)), Gaussian source."""
    deg, cells, dt = 3, (6, 6, 6), 5e-4
    o = O.Oracle(deg, cells, perturb=0.1, seed=5)
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), dt)
    q = o.gaussian_source(50.0, (0.5, 0.5, 0.9), 0.1)
    T_old = np.zeros(o.n_dofs)
    T_prev = o.distribute(np.random.default_rng(1).uniform(0, 1, o.n_dofs))
    # oracle: predictor = T_prev (first step), linearise there, solve to 1e-12
    Tg = T_prev.copy()
    r = o.create_rhs(Tg, T_prev, q)
    d, its, _ = o.cg(r, T_lin=Tg, T_old=T_prev, rel_tol=1e-13)
    T_ref = Tg + d
    op = H.HeatDiffuseOperator(H.box_mesh(deg, cells, perturb=0.1, seed=5))
    op.set_material(H.material(law=1, k=1.0, k1=0.5))
    lin = H.LinearSolverData(preconditioner_type=precond, rel_tolerance=1e-10)
    opn = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_NONE, single_linearization=True)
    opn.set_initial_condition(torch.tensor(T_prev, device="cuda"))
    opn.heat_source = torch.tensor(q, device="cuda")
    st = opn.solve(dt)
    T = opn.T.cpu().numpy()
    assert np.abs(T - T_ref).max() <= 1e-7 * np.abs(T_ref).max()
    assert np.array_equal(opn.T_old.cpu().numpy(), T_prev)
    assert st.linear_iterations > 0


def test_cpu_correctness_case_matches_oracle():
    """The small CPU-runnable case: FE_Q(2) on 16^3 cells (35,937 DoFs), k = rho cp = 1,
    dt = 1e-3, Dirichlet 0 on all faces, T0 ~ U[0, 1] (seeded; constrained DoFs set to
    0), nodally interpolated source exp(-|x - c|^2 / 0.1^2) at c = (0.5, 0.5, 0.9), one
    Jacobi-CG solve to 1e-10 relative, against the oracle's step."""
    deg, cells, dt = 2, (16, 16, 16), 1e-3
    o = O.Oracle(deg, cells)
    o.set_material(O.material(O.LAW_CONSTANT, k=1.0), dt)
    q = o.gaussian_source(1.0, (0.5, 0.5, 0.9), 0.1)
    T0 = o.distribute(np.random.default_rng(1).uniform(0, 1, o.n_dofs))
    r = o.create_rhs(T0, T0, q)
    d, _, _ = o.cg(r, T_lin=T0, T_old=T0, rel_tol=1e-13)
    T_ref = T0 + d
    op = H.HeatDiffuseOperator(H.box_mesh(deg, cells))
    op.set_material(H.material(law=0, k=1.0))
    opn = H.HeatDiffuseOperation(op, H.LinearSolverData(rel_tolerance=1e-10),
                                 predictor=L.PREDICTOR_NONE, single_linearization=True)
    opn.set_initial_condition(torch.tensor(T0, device="cuda"))
    opn.heat_source = torch.tensor(q, device="cuda")
    st = opn.solve(dt)
    T = opn.T.cpu().numpy()
    assert op.n_dofs == 35937
    assert np.abs(T - T_ref).max() <= 1e-7 * np.abs(T_ref).max()
    assert 0 < st.linear_iterations < 200


# applications/mp-heat-transfer/cases/solidification_slab/tests/solidification_slab.mpirun=1.output
SLAB = [2.82611e+02, 2.82458e+02, 2.82345e+02, 2.82252e+02, 2.82169e+02]


def test_solidification_slab_newton_gmres_on_gpu():
    """The reference's liquid-solid regression case through the GPU Newton path with the
    reference's default linear solver (GMRES, Jacobi), 1D slab as a one-cell-thick 3D mesh."""
    op = H.HeatDiffuseOperator(H.box_mesh(1, (128, 1, 1), dirichlet=("x-",),
                                          dirichlet_values={"x-": 253.0}))
    op.set_material(H.material(law=L.LAW_LIQUID_SOLID, rho=1000.0, cp=4226.0, k=0.556,
                               rho_s=1000.0, cp_s=1762.0, k_s=2.22, T_solidus=270.0,
                               T_liquidus=276.0))
    lin = H.LinearSolverData(solver_type=L.SOLVER_GMRES, rel_tolerance=1e-12)
    opn = H.HeatDiffuseOperation(op, lin, H.NonlinearSolverData(residual_tolerance=1e-8))
    opn.set_initial_condition(torch.full((op.n_dofs,), 283.0, dtype=torch.float64, device="cuda"))
    for ref in SLAB:
        st = opn.solve(200.0)
        assert st.converged == 1
        assert float(f"{op.l2_norm(opn.T):.5e}") == ref


def test_unidirectional_heat_transfer_gmres_on_gpu():
    op = H.HeatDiffuseOperator(H.box_mesh(1, (32, 32, 1), (0, 0, 0), (0.1, 0.1, 1.0),
                                          dirichlet=()))
    op.set_material(H.material())
    opn = H.HeatDiffuseOperation(op, H.LinearSolverData(solver_type=L.SOLVER_GMRES,
                                                        rel_tolerance=1e-12),
                                 H.NonlinearSolverData(residual_tolerance=5e-9))
    opn.set_initial_condition(op.support_points()[:, 0].contiguous())
    for ref in UNIDIRECTIONAL:
        opn.solve(1e-4)
        assert float(f"{op.l2_norm(opn.T):.5e}") == ref


ROBIN = {
    "convection": (dict(convection=(25.0, 300.0)),
                   [1.00000e+02, 9.99999e+01, 9.99999e+01, 9.99998e+01, 9.99998e+01]),
    "radiation": (dict(radiation=(0.98, 300.0)),
                  [9.99998e+01, 9.99997e+01, 9.99995e+01, 9.99994e+01, 9.99992e+01]),
    "radiation_and_convection": (dict(convection=(25.0, 300.0), radiation=(0.98, 300.0)),
                                 [9.99998e+01, 9.99996e+01, 9.99994e+01, 9.99992e+01,
                                  9.99990e+01]),
}


@pytest.mark.parametrize("case", list(ROBIN))
def test_unidirectional_robin_on_gpu(case):
    """unidirectional_heat_transfer_with_* regression outputs through the GPU Newton +
    GMRES path with the Robin terms on the right boundary."""
    bc, refs = ROBIN[case]
    op = H.HeatDiffuseOperator(H.box_mesh(1, (32, 32, 1), (0, 0, 0), (0.1, 0.1, 1.0),
                                          dirichlet=()))
    op.set_material(H.material(rho=7850.0, cp=460.0, k=55.563))
    op.set_boundary("x+", **bc)
    opn = H.HeatDiffuseOperation(op, H.LinearSolverData(solver_type=L.SOLVER_GMRES,
                                                        rel_tolerance=1e-12),
                                 H.NonlinearSolverData(residual_tolerance=5e-9))
    opn.set_initial_condition(torch.full((op.n_dofs,), 1000.0, dtype=torch.float64,
                                         device="cuda"))
    for ref in refs:
        st = opn.solve(0.01)
        assert st.converged == 1
        assert float(f"{op.l2_norm(opn.T):.5e}") == ref


@pytest.mark.parametrize("precond", [L.PRECOND_JACOBI, L.PRECOND_MG_F32])
def test_host_buffer_step_matches_device_step(precond):
    """mpdg_heat_time_step_host (pinned host T, T_old and source; its copies overlap the
    step) gives the fields of mpdg_heat_time_step on device vectors, two steps in a row,
    with the history committed on the host side as well."""
    import ctypes as C
    op = H.HeatDiffuseOperator(H.box_mesh(3, (8, 8, 8)))
    op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
    lin = H.LinearSolverData(preconditioner_type=precond, rel_tolerance=1e-10,
                             abs_tolerance=0.0, cheb_picard=True)
    dev = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    N, dt = op.n_dofs, 5e-4
    T0 = torch.rand(N, dtype=torch.float64, device="cuda", generator=torch.Generator(
        device="cuda").manual_seed(3))
    op.distribute_constraints(T0)
    dev.set_initial_condition(T0.clone())
    hT = T0.cpu().pin_memory()
    hTo = T0.cpu().pin_memory()
    hq = torch.empty(N, dtype=torch.float64).pin_memory()
    q = op.new_vector()
    dev.heat_source = q
    for s in range(2):
        op.gaussian_source(q, 200.0, (0.3 + 0.1 * s, 0.5, 0.9), 0.1)
        hq.copy_(q)
        dev.solve(dt)
        step = L.StepStats()
        H.check(op._L.mpdg_heat_time_step_host(op.h, C.byref(dev.params), dt,
                                                0.0 if s == 0 else dt,
                                                C.c_void_p(hT.data_ptr()),
                                                C.c_void_p(hTo.data_ptr()),
                                                C.c_void_p(hq.data_ptr()), C.byref(step)))
        # equal up to the solver tolerance (the atomic scatter makes sums order-dependent)
        ref, ref_old = dev.T.cpu(), dev.T_old.cpu()
        assert (hT - ref).abs().max() <= 1e-8 * ref.abs().max()
        assert (hTo - ref_old).abs().max() <= 1e-8 * ref_old.abs().max()
        assert ref.abs().max() > 0.0


@pytest.mark.parametrize("cells,perturb", [((6, 4, 5), 0.2), ((4, 4, 3), 0.0)])
@pytest.mark.parametrize("precond", [L.PRECOND_JACOBI, L.PRECOND_MG_F32])
def test_host_buffer_steps_with_slab_upload_match_device_step(cells, perturb, precond):
    """The host-buffer steps upload the source in z-slabs and apply the residual to the cells of
    each slab as it arrives (sub-boxes of the mesh, their z faces Dirichlet only at the mesh's
    ends): on a deformed mesh with an odd number of cell layers and a Robin face, and on a mesh
    with fewer layers than slabs, the stateless and the resident steps follow the device step."""
    import ctypes as C
    mesh = H.box_mesh(3, cells, perturb=perturb, seed=6,
                      dirichlet=("x-", "y-", "y+", "z-", "z+"))
    op = H.HeatDiffuseOperator(mesh)
    op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
    op.set_boundary(1, convection=(5.0, 0.2))
    lin = H.LinearSolverData(preconditioner_type=precond, rel_tolerance=1e-10,
                             abs_tolerance=0.0, cheb_picard=True)
    dev = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    res = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    N, dt = op.n_dofs, 5e-4
    T0 = torch.rand(N, dtype=torch.float64, device="cuda", generator=torch.Generator(
        device="cuda").manual_seed(8))
    op.distribute_constraints(T0)
    dev.set_initial_condition(T0.clone())
    res.load_history_host(T0.cpu().contiguous(), T0.cpu().contiguous())
    hT, hTo = T0.cpu().pin_memory(), T0.cpu().pin_memory()
    hq = torch.empty(N, dtype=torch.float64).pin_memory()
    hR = torch.empty(N, dtype=torch.float64).pin_memory()
    q = op.new_vector()
    dev.heat_source = q
    for s in range(2):
        op.gaussian_source(q, 200.0, (0.4, 0.5, 0.2 + 0.5 * s), 0.2)
        hq.copy_(q)
        dev.solve(dt)
        step = L.StepStats()
        H.check(op._L.mpdg_heat_time_step_host(op.h, C.byref(dev.params), dt,
                                                0.0 if s == 0 else dt,
                                                C.c_void_p(hT.data_ptr()),
                                                C.c_void_p(hTo.data_ptr()),
                                                C.c_void_p(hq.data_ptr()), C.byref(step)))
        res.solve_resident(dt, hq, hR)
        ref = dev.T.cpu()
        assert ref.abs().max() > 0.0
        assert (hT - ref).abs().max() <= 1e-8 * ref.abs().max()
        assert (hR - ref).abs().max() <= 1e-8 * ref.abs().max()


@pytest.mark.parametrize("precond", [L.PRECOND_JACOBI, L.PRECOND_MG_F32,
                                     L.PRECOND_CHEBYSHEV_JACOBI_F32])
def test_resident_history_step_matches_device_step(precond):
    """mpdg_heat_time_step_resident (history on the device, pinned host source in, new T
    out) follows mpdg_heat_time_step on device vectors over three steps; store_history
    returns both history vectors, and the T the step downloaded (with the mixed-precision
    solvers as soon as the increment converged, during the residual recheck) equals the
    resident T bit for bit."""
    op = H.HeatDiffuseOperator(H.box_mesh(3, (8, 8, 8)))
    op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
    lin = H.LinearSolverData(preconditioner_type=precond, rel_tolerance=1e-10,
                             abs_tolerance=0.0, cheb_picard=True)
    dev = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    res = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    N, dt = op.n_dofs, 5e-4
    T0 = torch.rand(N, dtype=torch.float64, device="cuda", generator=torch.Generator(
        device="cuda").manual_seed(4))
    op.distribute_constraints(T0)
    dev.set_initial_condition(T0.clone())
    res.load_history_host(T0.cpu().contiguous(), torch.zeros(N, dtype=torch.float64))
    hq = torch.empty(N, dtype=torch.float64).pin_memory()
    hT = torch.empty(N, dtype=torch.float64).pin_memory()
    q = op.new_vector()
    dev.heat_source = q
    for s in range(3):
        op.gaussian_source(q, 200.0, (0.3 + 0.1 * s, 0.5, 0.9), 0.1)
        hq.copy_(q)
        dev.solve(dt)
        res.solve_resident(dt, hq, hT)
        ref = dev.T.cpu()
        assert (hT - ref).abs().max() <= 1e-8 * ref.abs().max()
    T_back = torch.empty(N, dtype=torch.float64)
    To_back = torch.empty(N, dtype=torch.float64)
    res.store_history_host(T_back, To_back)
    assert torch.equal(T_back, hT)
    ref_old = dev.T_old.cpu()
    assert (To_back - ref_old).abs().max() <= 1e-8 * ref_old.abs().max()
    # a step without a source and without a copy back
    res.solve_resident(dt)


def test_resident_step_needs_a_loaded_history():
    op = H.HeatDiffuseOperator(H.box_mesh(2, (4, 4, 4)))
    res = H.HeatDiffuseOperation(op)
    with pytest.raises(H.ExcInvalidArgument):
        res.solve_resident(1e-3)


# unidirectional_heat_transfer_with_velocity / _with_two_phase / _with_two_phase_rho_times_cp
#   .mpirun=4.output: Robin terms on x = 0.1, dt = 1e-3, velocity (-0.01, 0), two-phase
#   cases on the heaviside smoothed_heaviside(0.05 - y, 0.01) (the oracle's known-answer
#   test states the setting)
TRANSPORT = {
    "velocity": (False, False, [1.00000e+02, 1.00000e+02, 9.99999e+01, 9.99999e+01, 9.99999e+01]),
    "two_phase": (True, False, [1.00000e+02, 9.99999e+01, 9.99999e+01, 9.99998e+01, 9.99997e+01]),
    "two_phase_rho_times_cp": (True, True,
                               [1.00000e+02, 9.99999e+01, 9.99999e+01, 9.99998e+01, 9.99998e+01]),
}


@pytest.mark.parametrize("case", list(TRANSPORT))
def test_unidirectional_transport_on_gpu(case):
    """The velocity / two-phase regression outputs through the GPU Newton + GMRES path."""
    two_phase, vs, refs = TRANSPORT[case]
    op = H.HeatDiffuseOperator(H.box_mesh(1, (32, 32, 1), (0, 0, 0), (0.1, 0.1, 1.0),
                                          dirichlet=()))
    if two_phase:
        op.set_material(H.material(law=L.LAW_GAS_LIQUID, rho=7850.0, cp=460.0, k=55.563,
                                   rho_g=3925.0, cp_g=230.0, k_g=27.7815, volume_specific=vs))
    else:
        op.set_material(H.material(rho=7850.0, cp=460.0, k=55.563))
    x = op.support_points()
    vel = torch.zeros((3, op.n_dofs), dtype=torch.float64, device="cuda")
    vel[0] = -0.01
    d = 0.05 - x[:, 1]
    eps = 0.01
    hs = torch.where(d > eps, torch.ones_like(d), torch.where(
        d <= -eps, torch.zeros_like(d), (d + eps) / (2 * eps) + torch.sin(np.pi * d / eps) / (2 * np.pi)))
    op.set_fields(hs.contiguous() if two_phase else None, vel)
    op.set_boundary("x+", convection=(25.0, 300.0), radiation=(0.98, 300.0))
    opn = H.HeatDiffuseOperation(op, H.LinearSolverData(solver_type=L.SOLVER_GMRES,
                                                        rel_tolerance=1e-12),
                                 H.NonlinearSolverData(residual_tolerance=1e-6))
    opn.set_initial_condition(torch.full((op.n_dofs,), 1000.0, dtype=torch.float64,
                                         device="cuda"))
    for i, ref in enumerate(refs):
        st = opn.solve(1e-3)
        assert st.converged == 1
        norm = op.l2_norm(opn.T)
        if case == "two_phase_rho_times_cp" and i == 4:
            # 1.1e-9 relative below the rounding boundary of the printed value (the oracle
            # lands on the same 99.99974989)
            assert abs(norm - ref) <= 0.5e-4 + 2e-7, norm
        else:
            assert float(f"{norm:.5e}") == ref


# _with_velocity_and_solidification / _with_two_phase_and_solidification.mpirun=4.output (the
# oracle's known-answer test states the setting): liquid-solid and three-phase laws with a
# velocity, the second on a heaviside that moves with the velocity
SOLIDIFICATION_TRANSPORT = {
    "velocity_and_solidification": (0.01, 0.005, False,
                                    [1.97002e+02, 1.97003e+02, 1.97004e+02, 1.97005e+02,
                                     1.97006e+02]),
    "two_phase_and_solidification": (1.0, 1e-4, True,
                                     [1.96996e+02, 1.96992e+02, 1.96987e+02, 1.96983e+02,
                                      1.96979e+02]),
}


@pytest.mark.parametrize("precond", [L.PRECOND_JACOBI, L.PRECOND_CHEBYSHEV_JACOBI_F32])
@pytest.mark.parametrize("case", list(SOLIDIFICATION_TRANSPORT))
def test_unidirectional_solidification_with_transport_on_gpu(case, precond):
    """Also through GMRES with the FP32 Chebyshev-Jacobi preconditioner (flexible GMRES)."""
    dt, vel, two_phase, refs = SOLIDIFICATION_TRANSPORT[case]
    op = H.HeatDiffuseOperator(H.box_mesh(1, (32, 32, 1), (0, 0, 0), (0.1, 0.1, 1.0),
                                          dirichlet=()))
    ls = dict(rho=7850.0, cp=460.0, k=55.563, rho_s=7850.0, cp_s=700.0, k_s=17.0,
              T_solidus=1966.0, T_liquidus=1974.0)
    if two_phase:
        op.set_material(H.material(law=L.LAW_GAS_LIQUID_SOLID, rho_g=3925.0, cp_g=230.0,
                                   k_g=27.7815, sharp_gas_liquid=True, **ls))
    else:
        op.set_material(H.material(law=L.LAW_LIQUID_SOLID, **ls))
    x = op.support_points()
    v = torch.zeros((3, op.n_dofs), dtype=torch.float64, device="cuda")
    v[0] = -vel
    opn = H.HeatDiffuseOperation(op, H.LinearSolverData(solver_type=L.SOLVER_GMRES,
                                                        preconditioner_type=precond,
                                                        rel_tolerance=1e-12),
                                 H.NonlinearSolverData(residual_tolerance=1e-7))
    opn.set_initial_condition((1960.0 + 20.0 * x[:, 0] / 0.1).contiguous())
    eps = 0.01
    for i, ref in enumerate(refs):
        d = 0.2 / 3 - x[:, 0] - vel * (i + 1) * dt
        hs = torch.where(d > eps, torch.ones_like(d), torch.where(
            d <= -eps, torch.zeros_like(d),
            (d + eps) / (2 * eps) + torch.sin(np.pi * d / eps) / (2 * np.pi))).contiguous()
        op.set_fields(hs if two_phase else None, v)
        st = opn.solve(dt)
        assert st.converged == 1
        assert float(f"{op.l2_norm(opn.T):.5e}") == ref


_GRAPH_CASE = r"""
import json, sys, torch
from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
op = H.HeatDiffuseOperator(H.box_mesh(3, (16, 16, 16)))
op.set_material(H.material(law=L.LAW_LINEAR_K, k=1.0, k1=0.5))
out = {}
for name, pre in [("mg", L.PRECOND_MG_F32), ("cheb", L.PRECOND_CHEBYSHEV_JACOBI_F32)]:
    lin = H.LinearSolverData(preconditioner_type=pre, rel_tolerance=1e-10, abs_tolerance=0.0,
                             cheb_picard=True)
    opn = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR, single_linearization=True)
    q = op.new_vector()
    opn.heat_source = q
    its = []
    for s in range(3):
        op.gaussian_source(q, 300.0, (0.3 + 0.1 * s, 0.5, 0.9), 0.1)
        its.append(opn.solve(5e-4).linear_iterations)
    out[name] = {"its": its, "T": opn.T.cpu().tolist()}
out["launches"] = op.counters()["launches"]
json.dump(out, open(sys.argv[1], "w"))
"""


def test_graph_replay_matches_direct_launches(tmp_path):
    """The mixed-precision solvers replay one recorded iteration as a CUDA graph; with
    MPDG_GRAPHS=0 they launch directly. Both give the same iterations, fields (to the
    solver tolerance: the atomic scatter's summation order varies) and launch counts.
    Child processes, because the mode is read once per process."""
    import json
    import os
    import subprocess
    import sys
    res = {}
    for mode in ("1", "0"):
        path = tmp_path / f"graphs_{mode}.json"
        r = subprocess.run([sys.executable, "-c", _GRAPH_CASE, str(path)],
                           env=dict(os.environ, MPDG_GRAPHS=mode), capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        res[mode] = json.load(open(path))
    for name in ("mg", "cheb"):
        a, b = res["1"][name], res["0"][name]
        assert a["its"] == b["its"] and min(a["its"]) > 0
        Ta, Tb = torch.tensor(a["T"]), torch.tensor(b["T"])
        assert (Ta - Tb).abs().max() <= 1e-8 * Tb.abs().max()
    assert res["1"]["launches"] == res["0"]["launches"] > 0


# applications/mp-heat-transfer/cases/melt_front_propagation/tests/
#   melt_front_propagation_static_gusarov.mpirun=4.output
GUSAROV = [3.46470e-01, 3.46530e-01, 3.46591e-01, 3.46653e-01, 3.46715e-01]


@pytest.mark.parametrize("fused", [False, True])
def test_melt_front_propagation_static_gusarov_on_gpu(fused):
    """The reference's Gusarov laser case (2D Q1 96 x 32 on [0, 6e-4] x [-2e-4, 0], liquid-solid
    steel, Dirichlet 1000 at x_max, dt 5e-6) through the GPU Newton path (GMRES, the heat
    default), the source computed on the device with the planar Gusarov profile."""
    op = H.HeatDiffuseOperator(H.box_mesh(1, (96, 1, 32), (0, 0, -2e-4), (6e-4, 1.0, 0.0),
                                          dirichlet=("x+",), dirichlet_values={"x+": 1000.0}))
    op.set_material(H.material(law=L.LAW_LIQUID_SOLID, rho=7850.0, cp=460.0, k=55.563,
                               rho_s=7850.0, cp_s=700.0, k_s=17.0, T_solidus=1966.0,
                               T_liquidus=1974.0))
    laser = dict(radius=6e-5, gusarov=(0.7, 6e4, 5e-5), planar=True)
    lin = H.LinearSolverData(solver_type=L.SOLVER_GMRES, rel_tolerance=1e-12)
    opn = H.HeatDiffuseOperation(op, lin, H.NonlinearSolverData(residual_tolerance=1e-8))
    opn.set_initial_condition(torch.full((op.n_dofs,), 1000.0, dtype=torch.float64,
                                         device="cuda"))
    if fused:  # the source evaluated inside the residual kernel
        op.set_laser(L.LASER_GUSAROV, 5.0, (0.0, 0.5, 0.0), **laser)
    else:      # the nodal source vector, as LaserHeatSourceVolumetric fills it
        opn.heat_source = op.laser_source(op.new_vector(), L.LASER_GUSAROV, 5.0, (0.0, 0.5, 0.0),
                                          **laser)
    for ref in GUSAROV:
        st = opn.solve(5e-6)
        assert st.converged == 1
        assert float(f"{op.l2_norm(opn.T):.5e}") == ref


@pytest.mark.parametrize("fused", [False, True])
def test_moving_ramped_laser_steps_match_oracle(fused):
    """A Gauss volumetric laser moving along x (LaserOperation: scan speed 2, power ramped over
    the first two steps), 4 single-linearisation steps of the constant-k problem on a deformed
    FE_Q(2) mesh: the source as a nodal vector (compute_heat_source) or evaluated inside the
    residual kernel (attach), against the oracle's steps with its own laser source at the same
    positions and powers."""
    from meltpooldg_b200.laser import LaserData, LaserOperation
    deg, cells, dt = 2, (6, 5, 4), 0.05
    o = O.Oracle(deg, cells, perturb=0.15, seed=2)
    o.set_material(O.material(O.LAW_CONSTANT, k=0.3), dt)
    op = H.HeatDiffuseOperator(H.box_mesh(deg, cells, perturb=0.15, seed=2))
    op.set_material(H.material(law=0, k=0.3))
    data = LaserData(intensity_profile=L.LASER_GAUSS_VOLUMETRIC, power=20.0, radius=0.2,
                     power_over_time="ramp", power_start_time=0.0, power_end_time=0.1,
                     scan_speed=2.0, starting_position=(0.2, 0.5, 0.8))
    las = LaserOperation(data, op)
    las.reset(0.0)
    lin = H.LinearSolverData(rel_tolerance=1e-12)
    opn = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_NONE, single_linearization=True)
    T = np.zeros(o.n_dofs)
    opn.set_initial_condition(torch.tensor(T, device="cuda"))
    q = op.new_vector()
    for _ in range(4):
        las.move_laser(dt)
        if fused:
            opn.heat_source = None
            las.attach()
        else:
            opn.heat_source = las.compute_heat_source(q)
        opn.solve(dt)
        qo = o.laser_source(L.LASER_GAUSS_VOLUMETRIC, las.get_laser_power(),
                            las.get_laser_position(), radius=0.2)
        r = o.create_rhs(T, T, qo)
        d, _, _ = o.cg(r, T_lin=T, T_old=T, rel_tol=1e-13)
        T = T + d
    assert las.get_laser_position()[0] == pytest.approx(0.2 + 2.0 * 4 * dt)
    Tg = opn.T.cpu().numpy()
    assert np.abs(T).max() > 0.0
    assert np.abs(Tg - T).max() <= 1e-9 * np.abs(T).max()
