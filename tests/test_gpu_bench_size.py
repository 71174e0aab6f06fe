"""GPU parity against the oracle at the benchmark's sizes.

The cell kernels run persistent grids (occupancy x SM count CTAs) that loop over cell
batches and prefetch the next batch into L2; on the small meshes of the other parity tests
each CTA handles at most one batch. Here every CTA loops: 48^3 cells (110,592 cells, more than
ten batches per CTA at p = 3), 40^3 cells on a deformed mesh, and the benchmark mesh itself,
FE_Q(3) on 128^3 cells (57,066,625 DoFs). The kernels checked are the ones the benchmark step
launches: the FP64 k(T) tangent from its per-point fields (k_vmult2 LAW 7), the FP32 Picard
operator of the multigrid smoothers (k_vmult_picard_tc on the tensor cores, and the CUDA-core
k_vmult2 LAW 3) and its diagonal (k_diag_picard), the
FP64 inverse diagonal (k_diag) and the residual (k_rhs2) with the Gaussian source of the
benchmark, and the FE L2 norm (its multi-batch reduction).

Tolerances: FP64 1e-12 relative (max norm against max |oracle|), FP32 2e-5 relative, the
TF32 tensor-core operator 5e-3; the
implicit step 1e-6 relative (L2 and max) against the oracle's FP64 Jacobi-CG solution, the
accuracy the mixed-precision solver is specified to.
"""
import numpy as np
import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64, TOL32, TOL_STEP = 1e-12, 2e-5, 1e-6
TOL_TF32 = 5e-3  # the tensor-core Picard operator: TF32 operands
DT = 5e-4
LAW = dict(law=L.LAW_LINEAR_K, rho=1.0, cp=1.0, k=1.0, k1=0.5)  # k(T) = 1 + 0.5 T


def cuda(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def rel(a, b):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().double().numpy()
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def smooth_state(o, scale=1.0):
    """A smooth temperature field of the scale the benchmark reaches (T = O(1)), with a
    seeded random perturbation, Dirichlet values applied."""
    x = o.support_points()
    rng = np.random.default_rng(11)
    T = scale * (np.sin(np.pi * x[:, 0]) * np.sin(np.pi * x[:, 1]) * np.sin(np.pi * x[:, 2])
                 + 0.3 * np.exp(-((x[:, 0] - 0.4) ** 2 + (x[:, 1] - 0.5) ** 2 +
                                  (x[:, 2] - 0.95) ** 2) / 0.05 ** 2))
    T += 0.01 * rng.uniform(-1, 1, o.n_dofs)
    return o.distribute(T)


def pair(cells, perturb=0.0, seed=3, degree=3):
    o = O.Oracle(degree, cells, perturb=perturb, seed=seed)
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), DT)
    g = H.HeatDiffuseOperator(H.box_mesh(degree, cells, perturb=perturb, seed=seed))
    g.set_material(H.material(**LAW))
    g.reset_time_increment(DT)
    return o, g


def check_bench_kernels(o, g, tol64=TOL64):
    N = o.n_dofs
    rng = np.random.default_rng(5)
    src = rng.uniform(-1, 1, N)
    Tl = smooth_state(o)
    To = o.distribute(Tl - 0.02 * rng.uniform(0, 1, N))
    q = o.gaussian_source(500.0, (0.4, 0.5, 0.95), 0.05)
    Tl_d, To_d = cuda(Tl), cuda(To)
    g.set_linearization(Tl_d, To_d)
    # FP64 tangent (LAW 7 fields, built at this linearisation point)
    ref = o.vmult(src, Tl, To)
    assert rel(g.vmult(g.new_vector(), cuda(src)), ref) <= tol64
    # FP64 inverse diagonal
    dref = o.inverse_diagonal(Tl, To)
    dg = g.compute_inverse_diagonal_from_matrixfree(g.new_vector())
    assert rel(1.0 / dg.cpu().numpy(), 1.0 / dref) <= tol64
    del dref, dg
    # residual with the benchmark's source (accumulated into dst)
    base = rng.uniform(-1, 1, N)
    rref = o.create_rhs(Tl, To, q, dst=base.copy())
    rg = cuda(base)
    g.create_rhs(rg, To_d, cuda(q))
    assert rel(rg, rref) <= tol64
    del rref, rg, base
    # FP32 Picard operator and its inverse diagonal (the multigrid fine level)
    s32 = cuda(src, torch.float32)
    pref = o.vmult(src, Tl, To, form=2)
    g.set_picard_tensor_cores(True)  # the opt-in tensor-core kernel, where it exists
    tc = g.picard_tensor_cores
    g.set_picard_tensor_cores(False)
    assert rel(g.vmult_picard_f32(g.new_vector(torch.float32), s32), pref) <= TOL32
    if o.degree == 3:  # the same operator from the cell-row layout (the multigrid fine level)
        rows = torch.empty(g.cell_rows_size(), dtype=torch.float32, device="cuda")
        g.to_cell_rows_f32(rows, s32)
        assert rel(g.vmult_picard_f32_rows(g.new_vector(torch.float32), rows), pref) <= TOL32
        del rows
    if tc:  # the tensor-core kernel (opt-in) on the benchmark's mesh
        g.set_picard_tensor_cores(True)
        assert rel(g.vmult_picard_f32(g.new_vector(torch.float32), s32), pref) <= TOL_TF32
    del pref
    dpref = o.inverse_diagonal(Tl, To, form=2)
    dp = g.inverse_diagonal_picard_f32(g.new_vector(torch.float32))
    assert rel(1.0 / dp.cpu().double().numpy(), 1.0 / dpref) <= TOL32
    # FP32 exact tangent
    assert rel(g.vmult(g.new_vector(torch.float32), s32), ref) <= TOL32
    # FE L2 norm (multi-batch reduction)
    assert abs(g.l2_norm(Tl_d) - o.l2_norm(Tl)) <= 1e-13 * o.l2_norm(Tl)


def test_bench_kernels_multi_batch_affine_48cubed():
    o, g = pair((48, 48, 48))
    check_bench_kernels(o, g)


def test_bench_kernels_multi_batch_deformed_40cubed():
    o, g = pair((40, 40, 40), perturb=0.2, seed=8)
    check_bench_kernels(o, g)


@pytest.mark.parametrize("perturb", [0.0, 0.2])
def test_production_degree_kernels_multi_batch_40cubed(perturb):
    """FE_Q(4), the production run's degree (deformed +-0.2 h there): the line-per-thread FP64
    tangent, the register-resident FP32 operators and the diagonals, 4,173,281 DoFs."""
    o, g = pair((40, 40, 40), perturb=perturb, seed=8, degree=4)
    check_bench_kernels(o, g)


def test_bench_kernels_at_the_benchmark_size():
    """FE_Q(3) on 128^3 cells: the benchmark's mesh, operator and source."""
    o, g = pair((128, 128, 128))
    assert o.n_dofs == 57066625
    check_bench_kernels(o, g)


@pytest.mark.parametrize("precond", [L.PRECOND_MG_F32, L.PRECOND_CHEBYSHEV_JACOBI_F32])
def test_benchmark_step_at_48cubed_matches_oracle(precond):
    """One step of the benchmark problem (k = 1 + 0.5 T, dt = 5e-4, Dirichlet 0, Gaussian
    source r = 0.05 at z = 0.95) on 48^3 cells with the benchmark's solver (FP64 flexible CG
    with the FP32 p-multigrid, one linearisation, |b - J T| <= 1e-8 |b|), against the oracle's
    FP64 Jacobi-CG solution of the same linearised step solved to 1e-12: L2 and max error."""
    o, g = pair((48, 48, 48))
    T_prev = smooth_state(o, 0.5)
    q = o.gaussian_source(500.0, (0.4, 0.5, 0.95), 0.05)
    # oracle: linearise at the previous state (predictor none), solve to 1e-12
    r = o.create_rhs(T_prev, T_prev, q)
    d, its_ref, _ = o.cg(r, T_lin=T_prev, T_old=T_prev, rel_tol=1e-12)
    T_ref = T_prev + d
    lin = H.LinearSolverData(preconditioner_type=precond, rel_tolerance=1e-8, abs_tolerance=0.0,
                             cheb_degree=6, cheb_picard=True)
    opn = H.HeatDiffuseOperation(g, lin, predictor=L.PREDICTOR_NONE, single_linearization=True)
    opn.set_initial_condition(cuda(T_prev))
    opn.heat_source = cuda(q)
    st = opn.solve(DT)
    T = opn.T.cpu().numpy()
    e_l2 = np.linalg.norm(T - T_ref) / np.linalg.norm(T_ref)
    e_max = np.abs(T - T_ref).max() / np.abs(T_ref).max()
    print(f"48^3 step: {st.linear_iterations} outer iterations (oracle Jacobi-CG {its_ref}), "
          f"rel L2 {e_l2:.2e}, rel max {e_max:.2e}")
    assert e_l2 <= TOL_STEP and e_max <= TOL_STEP
    assert 0 < st.linear_iterations < its_ref
    # the fine level's iterate in cell rows exactly when the opt-in asks for it
    assert g.picard_cell_rows == (__import__("os").environ.get("MPDG_PICARD_ROWS") == "1")


def test_benchmark_step_with_cell_row_smoother_iterate():
    """The 48^3 benchmark step with the multigrid fine level's iterate kept in the cell-row
    layout (opt-in, MPDG_PICARD_ROWS=1) instead of the lexicographic one, in a child process
    because the choice is read once per process: the same oracle bounds, and the Chebyshev
    preconditioner on the same layout."""
    import os
    import subprocess
    import sys
    env = dict(os.environ, MPDG_PICARD_ROWS="1")
    here = os.path.dirname(__file__)
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p",
                        "no:cacheprovider", __file__,
                        os.path.join(here, "test_gpu_operator.py"), "-k",
                        "benchmark_step_at_48cubed or multigrid_mixed_precision_cg or "
                        "chebyshev_mixed_precision_cg"],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert " passed" in r.stdout


# the vmult sweep's small meshes (bench_vmult_sweep.py --size small, ~2 M DoFs each)
SWEEP_SMALL = {1: 125, 2: 62, 3: 42, 4: 31, 5: 25, 6: 21}


@pytest.mark.parametrize("degree", sorted(SWEEP_SMALL))
@pytest.mark.parametrize("perturb", [0.0, 0.2])
def test_vmult_sweep_meshes_match_oracle(degree, perturb):
    """The operator of the cfg2 sweep (M/dt + K, rho cp = k = 1, dt = 1e-3, seeded U[-1, 1]
    input) on its ~2 M-DoF meshes, where every CTA of the persistent grids loops: FP64 to 1e-12,
    FP32 to 2e-5 (2e-4 for p >= 5, as the small-mesh tests)."""
    m = SWEEP_SMALL[degree]
    o = O.Oracle(degree, (m,) * 3, perturb=perturb, seed=1)
    o.set_material(O.material(O.LAW_CONSTANT, k=1.0), 1e-3)
    g = H.HeatDiffuseOperator(H.box_mesh(degree, (m,) * 3, perturb=perturb, seed=1))
    g.set_material(H.material(law=L.LAW_CONSTANT, k=1.0))
    g.reset_time_increment(1e-3)
    z = g.new_vector()
    g.set_linearization(z, z)
    src = np.random.default_rng(degree).uniform(-1, 1, o.n_dofs)
    ref = o.vmult(src)
    assert rel(g.vmult(g.new_vector(), cuda(src)), ref) <= TOL64
    tol32 = TOL32 * (10 if degree >= 5 else 1)
    assert rel(g.vmult(g.new_vector(torch.float32), cuda(src, torch.float32)), ref) <= tol32
