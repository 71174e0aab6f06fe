"""GPU parity of the operator verbs against the CPU oracle (same seeded inputs).

Tolerances: FP64 verbs 1e-12 relative (max norm against max |oracle|); the FP32
operator 2e-5 relative.
"""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LAWS = {
    "constant": dict(law=0, rho=1.0, cp=1.0, k=1.0),
    "linear_k": dict(law=1, rho=1.0, cp=1.0, k=1.0, k1=0.5),
    "liquid_solid": dict(law=2, rho=1000.0, cp=4226.0, k=0.556, rho_s=900.0, cp_s=1762.0,
                         k_s=2.22, T_solidus=0.2, T_liquidus=0.8),
}
TOL64 = 1e-12
TOL32 = 2e-5
TOL_TF32 = 5e-3  # the tensor-core Picard operator: TF32 operands (10-bit mantissa)


def pair(degree, cells, perturb=0.0, law="constant", dt=1e-3, dirichlet=0x3F, lo=(0, 0, 0),
         hi=(1, 1, 1), values=(0.0,) * 6, seed=3):
    o = O.Oracle(degree, cells, lo=lo, hi=hi, perturb=perturb, seed=seed, dirichlet_mask=dirichlet,
                 dirichlet_value=values)
    o.set_material(O.material(**LAWS[law]), dt)
    faces = [f for f in range(6) if dirichlet & (1 << f)]
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, lo, hi, perturb, seed, faces,
                                         list(values)))
    g.set_material(H.material(**LAWS[law]))
    g.reset_time_increment(dt)
    return o, g


def cuda(a, dtype=torch.float64):
    return torch.tensor(a, dtype=dtype, device="cuda")


def rel(a, b):
    a = a.detach().cpu().numpy().astype(np.float64) if isinstance(a, torch.Tensor) else a
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("perturb", [0.0, 0.2])
@pytest.mark.parametrize("law", list(LAWS))
def test_vmult_diag_rhs_match_oracle(degree, perturb, law):
    cells = (5, 4, 3) if degree <= 4 else (3, 3, 2)
    o, g = pair(degree, cells, perturb, law)
    rng = np.random.default_rng(100 * degree + int(10 * perturb))
    N = o.n_dofs
    assert g.n_dofs == N and g.dims == o.dims
    src = rng.uniform(-1, 1, N)
    Tl = rng.uniform(0, 1, N)
    To = rng.uniform(0, 1, N)
    q = rng.uniform(0, 5, N)
    Tl_d, To_d = cuda(Tl), cuda(To)
    g.set_linearization(Tl_d, To_d)
    # FP64 vmult
    ref = o.vmult(src, Tl, To)
    dst = g.new_vector()
    g.vmult(dst, cuda(src))
    assert rel(dst, ref) <= TOL64
    # FP32 vmult (geometry, coefficients and linearisation point in FP32)
    d32 = g.new_vector(torch.float32)
    g.vmult(d32, cuda(src, torch.float32))
    assert rel(d32, ref) <= TOL32 * (10 if degree >= 5 else 1)
    # inverse diagonal
    dref = o.inverse_diagonal(Tl, To)
    dg = g.compute_inverse_diagonal_from_matrixfree(g.new_vector())
    assert rel(1.0 / dg.cpu().numpy(), 1.0 / dref) <= TOL64
    # create_rhs (dst is accumulated, not zeroed)
    base = rng.uniform(-1, 1, N)
    rref = o.create_rhs(Tl, To, q, dst=base.copy())
    rg = cuda(base)
    g.create_rhs(rg, To_d, cuda(q))
    assert rel(rg, rref) <= TOL64
    # L2 norm
    assert abs(g.l2_norm(Tl_d) - o.l2_norm(Tl)) <= 1e-13 * o.l2_norm(Tl)


@pytest.mark.parametrize("degree", [1, 2, 3, 4])
@pytest.mark.parametrize("cells", [(4, 3, 3), (3, 3, 3), (1, 2, 3)])
@pytest.mark.parametrize("perturb", [0.0, 0.2])
def test_fp32_operator_cell_pairs(degree, cells, perturb):
    """FP32 tangent and Picard operator against the oracle on meshes whose cell rows
    have even length (cells processed in adjacent pairs), odd length (pairs across
    rows) and an odd cell count (last pair half empty), with boundary-face terms."""
    o, g = pair(degree, cells, perturb, "linear_k", dirichlet=0b110000)
    for side, kw in ((0, dict(convection=(5.0, 300.0))), (3, dict(radiation=(0.5, 250.0)))):
        o.set_boundary(side, **kw)
        g.set_boundary(side, **kw)
    rng = np.random.default_rng(7 * degree + len(cells))
    N = o.n_dofs
    src, Tl, To = rng.uniform(-1, 1, N), rng.uniform(0.5, 1.5, N), rng.uniform(0.5, 1.5, N)
    g.set_linearization(cuda(Tl), cuda(To))
    s32 = cuda(src, torch.float32)
    assert rel(g.vmult(g.new_vector(torch.float32), s32), o.vmult(src, Tl, To)) <= TOL32
    ref = o.vmult(src, Tl, To, form=2)
    g.set_picard_tensor_cores(True)  # uniform box, FE_Q(3): the opt-in tensor-core kernel
    tc = g.picard_tensor_cores
    g.set_picard_tensor_cores(False)
    assert rel(g.vmult_picard_f32(g.new_vector(torch.float32), s32), ref) <= TOL32
    if tc:
        g.set_picard_tensor_cores(True)
        assert rel(g.vmult_picard_f32(g.new_vector(torch.float32), s32), ref) <= TOL_TF32
    dref = o.inverse_diagonal(Tl, To, form=2)
    dg = g.inverse_diagonal_picard_f32(g.new_vector(torch.float32))
    assert rel(1.0 / dg.cpu().double().numpy(), 1.0 / dref) <= TOL32


def test_fp32_packed_kernel_matches_oracle():
    """The packed-pair FP32 kernel (MPDG_FP32_PACKED=1) on the same cases, in a child
    process because the kernel choice is read once per process."""
    import os
    import subprocess
    import sys
    env = dict(os.environ, MPDG_FP32_PACKED="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p",
                        "no:cacheprovider", __file__, "-k", "fp32_operator_cell_pairs"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]


@pytest.mark.parametrize("mode", ["1", "0"])
def test_line_per_thread_tangent_fields_match_oracle(mode):
    """The line-per-thread FP64 k(T) tangent on deformed meshes at p >= 4 from the fields built
    once per linearisation at every degree (MPDG_TANGENT_FIELDS_LPT=1; the default takes them at
    p = 4 and 6) or at none (=0: T_lin evaluated in every application), on the same cases, in a
    child process because the choice is read once per process."""
    import os
    import subprocess
    import sys
    env = dict(os.environ, MPDG_TANGENT_FIELDS_LPT=mode)
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p",
                        "no:cacheprovider", __file__, "-k",
                        "vmult_diag_rhs_match_oracle and linear_k and 0.2 and (4 or 5 or 6)"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert " passed" in r.stdout


def test_register_kernel_geometry_preload_matches_oracle():
    """The register-resident operator on deformed meshes with its per-point geometry preloaded
    when the cell group starts for every eligible case (MPDG_GEO_PRELOAD_V2=1: FP32 and FP64,
    p <= 2, every law; the default preloads for FP64 p = 1 and the FP64 k(T) tangents at p = 2),
    on the same cases, in a child process because the choice is read once per process."""
    import os
    import subprocess
    import sys
    env = dict(os.environ, MPDG_GEO_PRELOAD_V2="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p",
                        "no:cacheprovider", __file__, "-k",
                        "(vmult_diag_rhs_match_oracle or fp32_operator_cell_pairs) and 0.2 and "
                        "(1 or 2)"],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert " passed" in r.stdout


def test_picard_operator_from_nodal_linearisation_point_matches_oracle():
    """The FP32 Picard operator with k(T_lin(q)) interpolated in the kernel from the gathered
    T_lin (MPDG_PICARD_NODAL=1) on the cell-pair meshes, and the benchmark step at 48^3 with
    the multigrid built on it, in a child process because the choice is read once per process."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(__file__)
    env = dict(os.environ, MPDG_PICARD_NODAL="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p",
                        "no:cacheprovider", __file__,
                        os.path.join(here, "test_gpu_bench_size.py"), "-k",
                        "fp32_operator_cell_pairs or benchmark_step_at_48cubed"],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert " passed" in r.stdout


@pytest.mark.parametrize("cells", [(4, 3, 3), (1, 2, 3), (5, 4, 3)])
@pytest.mark.parametrize("perturb", [0.0, 0.2])
@pytest.mark.parametrize("dirichlet", [0x3F, 0b110000, 0])
def test_picard_operator_from_cell_rows(cells, perturb, dirichlet):
    """The cell-row layout of FE_Q(3) (slot s of cell column c of x-row r holds node 3c + s,
    checked bit for bit) and the FP32 Picard operator applied from it: against the oracle's
    Picard form (2e-5) and the lexicographic kernel (1e-6, both FP32)."""
    o, g = pair(3, cells, perturb, "linear_k", dirichlet=dirichlet)
    rng = np.random.default_rng(sum(cells) + dirichlet)
    N = o.n_dofs
    src, Tl, To = rng.uniform(-1, 1, N), rng.uniform(0.5, 1.5, N), rng.uniform(0.5, 1.5, N)
    g.set_linearization(cuda(Tl), cuda(To))
    s32 = cuda(src, torch.float32)
    nd = [3 * c + 1 for c in cells]
    assert g.cell_rows_size() == 4 * cells[0] * nd[1] * nd[2]
    rows = torch.full((g.cell_rows_size(),), float("nan"), dtype=torch.float32, device="cuda")
    g.to_cell_rows_f32(rows, s32)
    lex = s32.cpu().numpy().reshape(nd[2] * nd[1], nd[0])
    expect = np.stack([lex[:, 3 * c:3 * c + 4] for c in range(cells[0])], axis=1).reshape(-1)
    assert np.array_equal(rows.cpu().numpy(), expect)
    y = g.vmult_picard_f32_rows(g.new_vector(torch.float32), rows)
    assert rel(y, o.vmult(src, Tl, To, form=2)) <= TOL32
    ylex = g.vmult_picard_f32(g.new_vector(torch.float32), s32)
    assert rel(y, ylex.cpu().double().numpy()) <= 1e-6


def test_cell_rows_reject_other_degrees_and_boundary_faces():
    _, g = pair(2, (2, 2, 2), 0.0, "linear_k")
    with pytest.raises(H.ExcNotImplemented):
        g.cell_rows_size()
    o, g = pair(3, (2, 2, 2), 0.0, "linear_k", dirichlet=0b110000)
    g.set_boundary(0, convection=(5.0, 300.0))
    g.set_linearization(g.new_vector(), g.new_vector())
    rows = torch.zeros(g.cell_rows_size(), dtype=torch.float32, device="cuda")
    with pytest.raises(H.ExcInvalidArgument):
        g.vmult_picard_f32_rows(g.new_vector(torch.float32), rows)


def test_picard_operator_rejects_other_laws():
    _, g = pair(2, (2, 2, 2), 0.0, "constant")
    g.set_linearization(g.new_vector(), g.new_vector())
    x = g.new_vector(torch.float32)
    with pytest.raises(H.ExcInvalidArgument):
        g.vmult_picard_f32(g.new_vector(torch.float32), x)


@pytest.mark.parametrize("planar", [False, True])
@pytest.mark.parametrize("profile", [0, 1, 2, 3])
@pytest.mark.parametrize("degree,perturb", [(2, 0.15), (3, 0.0)])
def test_laser_source_matches_oracle(profile, degree, perturb, planar):
    """The four volumetric laser intensity profiles at the support points against the
    oracle, on a box with the powder surface at z = 0 (Gusarov's convention)."""
    lo, hi, cells = (0, 0, -1), (1, 1, 0), (5, 4, 6)
    o = O.Oracle(degree, cells, lo=lo, hi=hi, perturb=perturb, seed=2)
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, lo, hi, perturb, 2))
    kw = dict(radius=0.4, direction=(0.0, 0.6, -0.8), gusarov=(0.55, 15.0, 0.4), planar=planar)
    ref = o.laser_source(profile, 25.0, (0.45, 0.5, 0.0), **kw)
    q = g.laser_source(g.new_vector(), profile, 25.0, (0.45, 0.5, 0.0), **kw)
    assert rel(q, ref) <= 1e-13
    assert np.abs(ref).max() > 0.0


@pytest.mark.parametrize("profile", [1, 3])
@pytest.mark.parametrize("degree,perturb,law", [(3, 0.0, "linear_k"), (2, 0.15, "constant"),
                                                (4, 0.1, "liquid_solid")])
def test_fused_laser_residual_equals_the_nodal_source_path(profile, degree, perturb, law):
    """create_rhs with the laser evaluated at the support points inside the residual kernel
    (mpdg_heat_set_laser, heat_source NULL) against create_rhs on the nodal source vector of
    mpdg_heat_laser_source, and against the oracle: the register-plane kernel (p <= 3,
    constant and linear-k laws) and the line-per-thread one (the rest)."""
    lo, hi, cells = (0, 0, -1), (1, 1, 0), (5, 4, 6)
    o = O.Oracle(degree, cells, lo=lo, hi=hi, perturb=perturb, seed=2)
    o.set_material(O.material(**LAWS[law]), 1e-3)
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, lo, hi, perturb, 2))
    g.set_material(H.material(**LAWS[law]))
    g.reset_time_increment(1e-3)
    kw = dict(radius=0.4, gusarov=(0.55, 15.0, 0.4))
    c = (0.45, 0.5, 0.0)
    rng = np.random.default_rng(degree)
    N = o.n_dofs
    T, To = rng.uniform(0, 1, N), rng.uniform(0, 1, N)
    g.set_linearization(cuda(T), cuda(To))
    q = g.laser_source(g.new_vector(), profile, 25.0, c, **kw)
    nodal = g.create_rhs(g.new_vector(), cuda(To), q)
    g.set_laser(profile, 25.0, c, **kw)
    fused = g.create_rhs(g.new_vector(), cuda(To), None)
    assert rel(fused, nodal.cpu().numpy()) <= 1e-14
    ref = o.create_rhs(T, To, o.laser_source(profile, 25.0, c, **kw))
    assert rel(fused, ref) <= TOL64
    g.set_laser(None)
    plain = g.create_rhs(g.new_vector(), cuda(To), None)
    assert rel(plain, o.create_rhs(T, To, None)) <= TOL64


def test_laser_source_rejects_bad_parameters():
    g = H.HeatDiffuseOperator(H.box_mesh(1, (2, 2, 2)))
    with pytest.raises(H.ExcInvalidArgument):
        g.laser_source(g.new_vector(), L.LASER_GAUSS_VOLUMETRIC, 1.0, (0.5, 0.5, 1.0), radius=0.0)
    with pytest.raises(H.ExcInvalidArgument):
        g.laser_source(g.new_vector(), L.LASER_GAUSS_PROJECTION, 1.0, (0.5, 0.5, 1.0), radius=0.1,
                       direction=(0.0, 0.0, -2.0))


@pytest.mark.parametrize("perturb", [0.0, 0.2])
def test_geometry_support_points_and_constraints(perturb):
    o, g = pair(3, (4, 3, 5), perturb, dirichlet=0b101101,
                values=(1.0, 2.0, 0.0, 3.0, 4.0, 5.0))
    x = g.support_points().cpu().numpy()
    assert np.abs(x - o.support_points()).max() <= 1e-14
    u = np.random.default_rng(1).uniform(size=o.n_dofs)
    ud = cuda(u)
    g.distribute_constraints(ud)
    assert np.array_equal(ud.cpu().numpy(), o.distribute(u.copy()))
    q = g.gaussian_source(g.new_vector(), 2.0, (0.5, 0.5, 0.9), 0.1)
    assert rel(q, o.gaussian_source(2.0, (0.5, 0.5, 0.9), 0.1)) <= 1e-14


def test_constrained_rows_and_zero_input():
    o, g = pair(2, (3, 3, 3), 0.1, "linear_k")
    N = o.n_dofs
    T = cuda(np.random.default_rng(2).uniform(size=N))
    g.set_linearization(T, T)
    dst = g.new_vector()
    g.vmult(dst, g.new_vector())
    assert torch.count_nonzero(dst) == 0
    src = cuda(np.random.default_rng(3).uniform(-1, 1, N))
    g.vmult(dst, src)
    mask = torch.tensor(o.mask().astype(bool), device="cuda")
    assert torch.count_nonzero(dst[mask]) == 0
    d = g.compute_inverse_diagonal_from_matrixfree(g.new_vector())
    assert torch.all(d[mask] == 1.0)


def test_single_cell_and_thin_meshes():
    for cells, degree in [((1, 1, 1), 1), ((1, 1, 1), 4), ((7, 1, 1), 2), ((1, 5, 2), 3)]:
        o, g = pair(degree, cells, 0.0, "liquid_solid", dirichlet=0)
        rng = np.random.default_rng(sum(cells))
        src, Tl, To = (rng.uniform(0, 1, o.n_dofs) for _ in range(3))
        g.set_linearization(cuda(Tl), cuda(To))
        dst = g.new_vector()
        g.vmult(dst, cuda(src))
        assert rel(dst, o.vmult(src, Tl, To)) <= TOL64


def test_errors_are_raised_not_silent():
    o, g = pair(2, (2, 2, 2))
    g.reset_time_increment(0.0)
    with pytest.raises(H.ExcZeroTimeIncrement):
        g.vmult(g.new_vector(), g.new_vector())
    g.reset_time_increment(1e-3)
    g.set_material(H.material(law=1, k1=0.5))
    with pytest.raises(H.ExcInvalidArgument):  # k(T) law without a linearisation point
        g.vmult(g.new_vector(), g.new_vector())
    with pytest.raises(H.ExcInvalidArgument):
        g.vmult(g.new_vector(), torch.zeros(g.n_dofs, dtype=torch.float64))  # host tensor
    with pytest.raises(H.ExcInvalidArgument):
        H.HeatDiffuseOperator(H.box_mesh(7, (2, 2, 2)))


@pytest.mark.parametrize("law", ["constant", "linear_k"])
def test_jacobi_cg_matches_oracle(law):
    o, g = pair(3, (6, 5, 4), 0.15, law, dt=1e-2)
    rng = np.random.default_rng(7)
    N = o.n_dofs
    Tl = rng.uniform(0, 1, N)
    b = o.vmult(rng.uniform(-1, 1, N), Tl, Tl)
    x_ref, its_ref, _ = o.cg(b, T_lin=Tl, T_old=Tl, rel_tol=1e-12)
    Tl_d = cuda(Tl)
    g.set_linearization(Tl_d, Tl_d)
    H.JacobiPreconditioner(g).update()
    x = g.new_vector()
    its = H.LinearSolver.solve(g, x, cuda(b), H.LinearSolverData(rel_tolerance=1e-12), True)
    assert abs(its - its_ref) <= 2
    assert rel(x, x_ref) <= 1e-9


@pytest.mark.parametrize("degree", [2, 3, 4])
def test_chebyshev_mixed_precision_cg(degree):
    o, g = pair(degree, (5, 5, 5), 0.2, "linear_k", dt=5e-3)
    rng = np.random.default_rng(degree)
    N = o.n_dofs
    Tl = rng.uniform(0, 1, N)
    b = o.vmult(rng.uniform(-1, 1, N), Tl, Tl)
    x_ref, its_ref, _ = o.cg(b, T_lin=Tl, T_old=Tl, rel_tol=1e-13)
    Tl_d = cuda(Tl)
    g.set_linearization(Tl_d, Tl_d)
    H.JacobiPreconditioner(g).update()
    x = g.new_vector()
    data = H.LinearSolverData(preconditioner_type=L.PRECOND_CHEBYSHEV_JACOBI_F32,
                              rel_tolerance=1e-10, cheb_degree=4)
    its = H.LinearSolver.solve(g, x, cuda(b), data, True)
    st = H.LinearSolver.last_stats
    assert st.true_residual <= 1e-10 * st.initial_residual * 1.0000001
    assert its < its_ref  # the polynomial preconditioner cuts outer iterations
    assert rel(x, x_ref) <= 1e-7


@pytest.mark.parametrize("picard", [False, True])
def test_chebyshev_mixed_precision_cg_larger_mesh(picard):
    """Flexible CG + FP32 Chebyshev on a 24^3-cell Q3 k(T) tangent at a smooth
    linearisation point: converges to the FP64 tolerance (true residual) in far fewer
    outer iterations than Jacobi-CG, with the exact FP32 tangent or the Picard operator
    in the preconditioner."""
    g = H.HeatDiffuseOperator(H.box_mesh(3, (24, 24, 24)))
    g.set_material(H.material(law=1, k=1.0, k1=0.5))
    g.reset_time_increment(5e-4)
    T = g.gaussian_source(g.new_vector(), 1.5, (0.5, 0.5, 0.8), 0.15)
    g.distribute_constraints(T)
    g.set_linearization(T, T)
    H.JacobiPreconditioner(g).update()
    x_src = g.gaussian_source(g.new_vector(), 1.0, (0.5, 0.5, 0.5), 0.2)
    g.distribute_constraints(x_src)  # homogeneous Dirichlet values
    b = g.vmult(g.new_vector(), x_src)
    its_j = H.LinearSolver.solve(g, g.new_vector(), b, H.LinearSolverData(rel_tolerance=1e-10),
                                 True)
    x = g.new_vector()
    data = H.LinearSolverData(preconditioner_type=L.PRECOND_CHEBYSHEV_JACOBI_F32,
                              rel_tolerance=1e-10, cheb_picard=picard)
    its_c = H.LinearSolver.solve(g, x, b, data, True)
    st = H.LinearSolver.last_stats
    assert st.true_residual <= 1e-10 * st.initial_residual * 1.0000001
    assert its_c * 2 < its_j, (its_c, its_j)
    assert torch.linalg.vector_norm(x - x_src) <= 1e-6 * torch.linalg.vector_norm(x_src)


@pytest.mark.parametrize("degree,cells,perturb,picard", [
    (3, (24, 24, 24), 0.0, True), (3, (24, 24, 24), 0.0, False), (2, (16, 24, 20), 0.15, True),
    (1, (32, 32, 32), 0.0, True), (4, (12, 12, 12), 0.2, True), (3, (16, 16, 16), 0.2, True)])
def test_multigrid_mixed_precision_cg(degree, cells, perturb, picard):
    """Flexible CG + FP32 p-multigrid V-cycle (FE_Q(p) -> FE_Q(1) -> h-coarsened FE_Q(1))
    on the k(T) tangent: converges to the FP64 tolerance (true residual) to the same
    solution in a mesh-independent handful of outer iterations (6-9 measured from 32^3
    to 128^3 cells), never more than the Chebyshev preconditioner needs + 2."""
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, perturb=perturb, seed=4))
    g.set_material(H.material(law=1, k=1.0, k1=0.5))
    g.reset_time_increment(5e-4)
    T = g.gaussian_source(g.new_vector(), 1.5, (0.5, 0.5, 0.8), 0.15)
    g.distribute_constraints(T)
    g.set_linearization(T, T)
    H.JacobiPreconditioner(g).update()
    x_src = g.gaussian_source(g.new_vector(), 1.0, (0.5, 0.5, 0.5), 0.2)
    g.distribute_constraints(x_src)
    b = g.vmult(g.new_vector(), x_src)
    cheb = H.LinearSolverData(preconditioner_type=L.PRECOND_CHEBYSHEV_JACOBI_F32,
                              rel_tolerance=1e-10, cheb_picard=picard, cheb_degree=6)
    its_c = H.LinearSolver.solve(g, g.new_vector(), b, cheb, True)
    x = g.new_vector()
    mg = H.LinearSolverData(preconditioner_type=L.PRECOND_MG_F32, rel_tolerance=1e-10,
                            cheb_picard=picard)
    its_m = H.LinearSolver.solve(g, x, b, mg, True)
    st = H.LinearSolver.last_stats
    assert st.true_residual <= 1e-10 * st.initial_residual * 1.0000001
    assert torch.linalg.vector_norm(x - x_src) <= 1e-6 * torch.linalg.vector_norm(x_src)
    assert its_m <= 12 and its_m <= its_c + 2, (its_m, its_c)


def test_multigrid_rejects_a_mesh_without_coarse_level():
    g = H.HeatDiffuseOperator(H.box_mesh(1, (5, 5, 5)))
    g.set_material(H.material(law=1, k=1.0, k1=0.5))
    g.reset_time_increment(1e-3)
    T = g.new_vector()
    g.set_linearization(T, T)
    H.JacobiPreconditioner(g).update()
    b = g.vmult(g.new_vector(), g.new_vector().fill_(1.0))
    with pytest.raises(H.ExcInvalidArgument):
        H.LinearSolver.solve(g, g.new_vector(), b,
                             H.LinearSolverData(preconditioner_type=L.PRECOND_MG_F32), True)


@pytest.mark.parametrize("restart", [5, 28])
def test_gmres_matches_oracle_on_nonsymmetric_tangent(restart):
    """Liquid-solid tangent at a rough linearisation point (strongly non-symmetric dk/dT
    term): right-preconditioned GMRES(m) against the oracle's GMRES."""
    law = dict(law=2, rho=1.0, cp=1.0, k=0.5, rho_s=1.2, cp_s=0.8, k_s=2.5, T_solidus=0.3,
               T_liquidus=0.7)
    o = O.Oracle(2, (5, 4, 4), perturb=0.1, seed=2)
    o.set_material(O.material(**law), 1e-2)
    g = H.HeatDiffuseOperator(H.box_mesh(2, (5, 4, 4), perturb=0.1, seed=2))
    g.set_material(H.material(**law))
    g.reset_time_increment(1e-2)
    rng = np.random.default_rng(11)
    N = o.n_dofs
    Tl = rng.uniform(0, 1, N)
    To = rng.uniform(0, 1, N)
    b = o.vmult(rng.uniform(-1, 1, N), Tl, To)
    x_ref, its_ref, _ = o.gmres(b, T_lin=Tl, T_old=To, rel_tol=1e-12, restart=restart)
    g.set_linearization(cuda(Tl), cuda(To))
    H.JacobiPreconditioner(g).update()
    x = g.new_vector()
    its = H.LinearSolver.solve(g, x, cuda(b), H.LinearSolverData(
        solver_type=L.SOLVER_GMRES, rel_tolerance=1e-12, gmres_restart=restart), True)
    assert abs(its - its_ref) <= max(2, its_ref // 10), (its, its_ref)
    assert rel(x, x_ref) <= 1e-9
    r = b - o.vmult(x.cpu().numpy(), Tl, To)
    assert np.linalg.norm(r) <= 1.01e-12 * np.linalg.norm(b)


@pytest.mark.parametrize("degree", [1, 2, 3, 4])
def test_boundary_terms_match_oracle(degree):
    """Convection + radiation on x-, radiation on z+, Neumann on x+, Dirichlet on y faces."""
    o, g = pair(degree, (4, 3, 3), 0.15, "linear_k", dirichlet=0b001100)
    for side, kw in ((0, dict(convection=(5.0, 300.0), radiation=(0.8, 320.0))),
                     (5, dict(radiation=(0.5, 250.0))), (1, dict(neumann=3.0))):
        o.set_boundary(side, **kw)
        g.set_boundary(side, **kw)
    rng = np.random.default_rng(degree)
    N = o.n_dofs
    src = rng.uniform(-1, 1, N)
    Tl = rng.uniform(0.5, 1.5, N)
    To = rng.uniform(0.5, 1.5, N)
    g.set_linearization(cuda(Tl), cuda(To))
    ref = o.vmult(src, Tl, To)
    assert rel(g.vmult(g.new_vector(), cuda(src)), ref) <= TOL64
    assert rel(g.vmult(g.new_vector(torch.float32), cuda(src, torch.float32)), ref) <= TOL32
    dref = o.inverse_diagonal(Tl, To)
    dg = g.compute_inverse_diagonal_from_matrixfree(g.new_vector())
    assert rel(1.0 / dg.cpu().numpy(), 1.0 / dref) <= TOL64
    rref = o.create_rhs(Tl, To)
    assert rel(g.create_rhs(g.new_vector(), cuda(To)), rref) <= TOL64
    with pytest.raises(H.ExcInvalidArgument):  # Neumann with convection on one face
        g.set_boundary(4, convection=(1.0, 0.0), neumann=1.0)


def test_cg_alpha_includes_boundary_terms():
    """CG with Robin terms: the fused p.Ap reduction must include the face part."""
    o, g = pair(2, (5, 4, 4), 0.1, "constant", dt=1e-2, dirichlet=0)
    o.set_boundary(1, convection=(50.0, 0.0))
    g.set_boundary(1, convection=(50.0, 0.0))
    rng = np.random.default_rng(3)
    b = o.vmult(rng.uniform(-1, 1, o.n_dofs))
    x_ref, its_ref, _ = o.cg(b, rel_tol=1e-12)
    g.set_linearization(g.new_vector(), g.new_vector())
    H.JacobiPreconditioner(g).update()
    x = g.new_vector()
    its = H.LinearSolver.solve(g, x, cuda(b), H.LinearSolverData(rel_tolerance=1e-12), True)
    assert abs(its - its_ref) <= 2
    assert rel(x, x_ref) <= 1e-9


def test_linear_solve_not_converged_raises():
    o, g = pair(3, (4, 4, 4), 0.0, dt=1.0)
    H.JacobiPreconditioner(g).update()
    b = cuda(np.random.default_rng(0).uniform(size=o.n_dofs))
    with pytest.raises(H.ExcNoConvergence):
        H.LinearSolver.solve(g, g.new_vector(), b,
                             H.LinearSolverData(max_iterations=3, rel_tolerance=1e-12), True)


TRANSPORT_CASES = {
    # law, material, heaviside, velocity
    "gas_liquid": (dict(law=3, rho=2.0, cp=3.0, k=5.0, rho_g=0.5, cp_g=1.5, k_g=0.3), True, False),
    "gas_liquid_sharp_vs": (dict(law=3, rho=2.0, cp=3.0, k=5.0, rho_g=0.5, cp_g=1.5, k_g=0.3,
                                 sharp_gas_liquid=True, volume_specific=True), True, False),
    "constant_velocity": (dict(law=0, rho=2.0, cp=3.0, k=5.0), False, True),
    "gas_liquid_velocity": (dict(law=3, rho=2.0, cp=3.0, k=5.0, rho_g=0.5, cp_g=1.5, k_g=0.3),
                            True, True),
    # temperature-dependent laws with the fields (kernel LAW 5): mushy zone inside the
    # sampled T range
    "liquid_solid_velocity": (dict(law=2, rho=1.0, cp=1.0, k=0.5, rho_s=1.2, cp_s=0.8, k_s=2.5,
                                   T_solidus=0.3, T_liquidus=0.7), False, True),
    "three_phase": (dict(law=4, rho=1.0, cp=1.0, k=0.5, rho_s=1.2, cp_s=0.8, k_s=2.5,
                         T_solidus=0.3, T_liquidus=0.7, rho_g=0.4, cp_g=1.5, k_g=0.2), True, False),
    "three_phase_sharp_vs_velocity": (dict(law=4, rho=1.0, cp=1.0, k=0.5, rho_s=1.2, cp_s=0.8,
                                           k_s=2.5, T_solidus=0.3, T_liquidus=0.7, rho_g=0.4,
                                           cp_g=1.5, k_g=0.2, sharp_gas_liquid=True,
                                           volume_specific=True), True, True),
}


def transport_pair(degree, cells, perturb, case, dt=1e-2):
    law, with_h, with_v = TRANSPORT_CASES[case]
    hi = (1.0, 1.3, 0.8)
    o = O.Oracle(degree, cells, hi=hi, perturb=perturb, seed=7)
    o.set_material(O.material(**law), dt)
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, (0, 0, 0), hi, perturb, 7))
    g.set_material(H.material(**law))
    g.reset_time_increment(dt)
    x = o.support_points()
    Hf = 0.5 + 0.5 * np.tanh((x[:, 0] - 0.45) / 0.1) if with_h else None
    V = np.stack([np.sin(3 * x[:, 1]), 0.5 + x[:, 2], -x[:, 0] * x[:, 1]]) if with_v else None
    o.set_fields(Hf, V)
    g.set_fields(None if Hf is None else cuda(Hf), None if V is None else cuda(V).contiguous())
    return o, g


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("perturb", [0.0, 0.2])
@pytest.mark.parametrize("case", list(TRANSPORT_CASES))
def test_two_phase_transport_matches_oracle(degree, perturb, case):
    """Gas-liquid law on the heaviside field and the convective term: FP64 vmult, inverse
    diagonal and residual to 1e-12, the FP32 operator to 2e-5 (x10 for p >= 5)."""
    cells = (5, 4, 3) if degree <= 4 else (3, 3, 2)
    o, g = transport_pair(degree, cells, perturb, case)
    rng = np.random.default_rng(7 * degree + int(10 * perturb))
    N = o.n_dofs
    src = rng.uniform(-1, 1, N)
    T, To, q = rng.uniform(0, 1, N), rng.uniform(0, 1, N), rng.uniform(0, 5, N)
    g.set_linearization(cuda(T), cuda(To))
    ref = o.vmult(src, T, To)
    dst = g.vmult(g.new_vector(), cuda(src))
    assert rel(dst, ref) <= TOL64
    d32 = g.vmult(g.new_vector(torch.float32), cuda(src, torch.float32))
    assert rel(d32, ref) <= TOL32 * (10 if degree >= 5 else 1)
    dref = o.inverse_diagonal(T, To)
    dg = g.compute_inverse_diagonal_from_matrixfree(g.new_vector())
    assert rel(1.0 / dg.cpu().numpy(), 1.0 / dref) <= TOL64
    base = rng.uniform(-1, 1, N)
    rref = o.create_rhs(T, To, q, dst=base.copy())
    rg = cuda(base)
    g.create_rhs(rg, cuda(To), cuda(q))
    assert rel(rg, rref) <= TOL64


def test_fields_are_rebuilt_after_set_fields_and_set_material():
    o, g = transport_pair(3, (4, 3, 3), 0.1, "gas_liquid_velocity")
    rng = np.random.default_rng(5)
    src = rng.uniform(-1, 1, o.n_dofs)
    g.vmult(g.new_vector(), cuda(src))
    x = o.support_points()
    Hf = 0.5 + 0.5 * np.tanh((x[:, 1] - 0.6) / 0.2)
    V = np.stack([0 * x[:, 0] + 1.0, x[:, 0], 0 * x[:, 0]])
    o.set_fields(Hf, V)
    g.set_fields(cuda(Hf), cuda(V).contiguous())
    assert rel(g.vmult(g.new_vector(), cuda(src)), o.vmult(src)) <= TOL64
    m = dict(law=3, rho=1.0, cp=4.0, k=2.0, rho_g=0.1, cp_g=1.0, k_g=0.5)
    o.set_material(O.material(**m), 1e-2)
    g.set_material(H.material(**m))
    assert rel(g.vmult(g.new_vector(), cuda(src)), o.vmult(src)) <= TOL64
    o.set_fields(Hf, None)
    g.set_fields(cuda(Hf), None)
    assert rel(g.vmult(g.new_vector(), cuda(src)), o.vmult(src)) <= TOL64


def test_gmres_on_the_convective_operator_matches_oracle():
    o, g = transport_pair(2, (6, 5, 4), 0.1, "gas_liquid_velocity", dt=1e-1)
    rng = np.random.default_rng(13)
    N = o.n_dofs
    b = o.vmult(rng.uniform(-1, 1, N))
    x_ref, its_ref, _ = o.gmres(b, rel_tol=1e-12, restart=28)
    g.set_linearization(cuda(np.zeros(N)), cuda(np.zeros(N)))
    H.JacobiPreconditioner(g).update()
    x = g.new_vector()
    its = H.LinearSolver.solve(g, x, cuda(b), H.LinearSolverData(
        solver_type=L.SOLVER_GMRES, rel_tolerance=1e-12), True)
    assert abs(its - its_ref) <= max(2, its_ref // 10), (its, its_ref)
    assert rel(x, x_ref) <= 1e-9


def test_fields_reject_unsupported_combinations():
    o, g = transport_pair(2, (4, 4, 4), 0.0, "constant_velocity")
    with pytest.raises(H.ExcInvalidArgument):
        g.set_material(H.material(law=1, k1=0.5))  # velocity with the linear-k law
    N = g.n_dofs
    g.set_linearization(cuda(np.zeros(N)), cuda(np.zeros(N)))
    H.JacobiPreconditioner(g).update()
    with pytest.raises(H.ExcInvalidArgument):
        H.LinearSolver.solve(g, g.new_vector(), cuda(np.ones(N)), H.LinearSolverData(
            preconditioner_type=L.PRECOND_MG_F32), True)
    g2 = H.HeatDiffuseOperator(H.box_mesh(2, (3, 3, 3)))
    g2.reset_time_increment(1e-2)
    z = g2.new_vector()
    g2.set_linearization(z, z)
    for law in (3, 4):  # gas-liquid laws without a heaviside
        g2.set_material(H.material(law=law, rho_g=0.5))
        with pytest.raises(H.ExcInvalidArgument):
            g2.vmult(g2.new_vector(), g2.new_vector())


@pytest.mark.parametrize("degree", [2, 3])
def test_tangent_fields_follow_the_linearisation_point(degree):
    """The three-phase operator's coefficient fields are rebuilt after set_linearization,
    reset_time_increment and set_fields (FP64 and FP32)."""
    o, g = transport_pair(degree, (4, 3, 3), 0.1, "three_phase_sharp_vs_velocity")
    rng = np.random.default_rng(21)
    N = o.n_dofs
    src = rng.uniform(-1, 1, N)
    for it in range(3):
        T, To = rng.uniform(0, 1, N), rng.uniform(0, 1, N)
        if it == 1:
            o.set_material(o._material, 3e-3)
            g.reset_time_increment(3e-3)
        if it == 2:
            x = o.support_points()
            Hf = 0.5 + 0.5 * np.tanh((x[:, 2] - 0.3) / 0.1)
            o.set_fields(Hf, None)
            g.set_fields(cuda(Hf), None)
        g.set_linearization(cuda(T), cuda(To))
        ref = o.vmult(src, T, To)
        assert rel(g.vmult(g.new_vector(), cuda(src)), ref) <= TOL64
        assert rel(g.vmult(g.new_vector(torch.float32), cuda(src, torch.float32)), ref) <= TOL32


@pytest.mark.parametrize("case", ["liquid_solid", "three_phase_sharp_vs_velocity"])
def test_flexible_gmres_with_fp32_chebyshev(case):
    """GMRES with the FP32 Chebyshev-Jacobi preconditioner (flexible: the preconditioned
    directions are stored) on nonsymmetric operators at a smooth linearisation point converges
    to the oracle's GMRES solution, to the FP64 tolerance, in fewer iterations than
    Jacobi-GMRES. (At a random linearisation point the dk/dT grad(T) term dominates, Jacobi-
    GMRES itself stalls and the Lanczos interval estimate breaks down.)"""
    if case == "liquid_solid":
        law = dict(law=2, rho=1.0, cp=1.0, k=0.5, rho_s=1.2, cp_s=0.8, k_s=2.5, T_solidus=0.3,
                   T_liquidus=0.7)
        o = O.Oracle(3, (6, 5, 5), perturb=0.1, seed=2)
        o.set_material(O.material(**law), 1e-2)
        g = H.HeatDiffuseOperator(H.box_mesh(3, (6, 5, 5), perturb=0.1, seed=2))
        g.set_material(H.material(**law))
        g.reset_time_increment(1e-2)
    else:
        o, g = transport_pair(3, (6, 5, 5), 0.1, case, dt=1e-2)
    rng = np.random.default_rng(17)
    N = o.n_dofs
    # a smooth linearisation point across the mushy zone (0.3 .. 0.7), as in a time step
    x = o.support_points()
    Tl = 0.5 + 0.3 * np.sin(3 * x[:, 0]) + 0.1 * np.cos(2 * x[:, 1])
    To = Tl - 0.05 * x[:, 2]
    b = o.vmult(rng.uniform(-1, 1, N), Tl, To)
    x_ref, _, _ = o.gmres(b, T_lin=Tl, T_old=To, rel_tol=1e-12, restart=28)
    g.set_linearization(cuda(Tl), cuda(To))
    H.JacobiPreconditioner(g).update()
    its = {}
    # restart 3: several restart cycles, each ending on a direction it does not precondition
    for name, pre, m in [("jacobi", L.PRECOND_JACOBI, 28),
                         ("cheb", L.PRECOND_CHEBYSHEV_JACOBI_F32, 28),
                         ("cheb_restart3", L.PRECOND_CHEBYSHEV_JACOBI_F32, 3)]:
        x = g.new_vector()
        its[name] = H.LinearSolver.solve(g, x, cuda(b), H.LinearSolverData(
            solver_type=L.SOLVER_GMRES, preconditioner_type=pre, rel_tolerance=1e-12,
            abs_tolerance=0.0, cheb_degree=6, gmres_restart=m), True)
        assert rel(x, x_ref) <= 1e-9, name
        r = b - o.vmult(x.cpu().numpy(), Tl, To)
        assert np.linalg.norm(r) <= 1.05e-12 * np.linalg.norm(b), name
    assert its["cheb"] < its["jacobi"], its
    assert its["cheb_restart3"] > 3, its
