"""The trained learned-guess model against linear extrapolation on a held-out scan path.

The guess scales the network's correction by the residual-minimising step length, so
its initial residual never exceeds the extrapolation's; the test records what the
network gains in initial residual and CG iterations (the solver still iterates to the
same 1e-8 tolerance, so the solution is unchanged)."""
import os

import pytest
import torch

from meltpooldg_b200 import _lib as L
from meltpooldg_b200 import heat as H
from meltpooldg_b200 import learned as LG

pytestmark = pytest.mark.gpu
MODEL = os.path.join(os.path.dirname(LG.__file__), "models", "heat_guess_p3_h96")


def run(op, model, seed, n_steps=14, direction=False):
    path = LG.scan_path(torch.Generator().manual_seed(seed))
    lin = H.LinearSolverData(preconditioner_type=L.PRECOND_CHEBYSHEV_JACOBI_F32,
                             rel_tolerance=1e-8, abs_tolerance=0.0, cheb_degree=6,
                             cheb_picard=True, cheb_eig_reuse=True)
    opn = H.HeatDiffuseOperation(op, lin, predictor=L.PREDICTOR_LINEAR,
                                 single_linearization=True)
    q = op.new_vector()
    opn.heat_source = q
    its, res = [], []
    for s in range(n_steps):
        op.gaussian_source(q, LG.AMP, path((s + 1) * LG.DT), LG.RADIUS)
        if model is not None and s > 0 and direction:
            opn.set_direction(model.direction(op, opn.T, opn.T_old, q, LG.DT))
            opn.params.predictor = L.PREDICTOR_LINEAR_DIRECTION
        elif model is not None and s > 0:
            g, _ = model.guess(op, opn.T, opn.T_old, q, LG.DT)
            opn.set_guess(g)
            opn.params.predictor = L.PREDICTOR_GIVEN
        else:
            opn.params.predictor = L.PREDICTOR_LINEAR
        st = opn.solve(LG.DT)
        its.append(st.linear_iterations)
        res.append(st.initial_relative_residual)
    return its, res, opn.T.clone()


def test_learned_guess_on_held_out_path():
    assert os.path.exists(MODEL + ".pt"), "trained model missing"
    op = LG.make_operator(32)
    model = LG.GuessModel.load(MODEL, stride=1)
    its0, res0, T0 = run(op, None, seed=99)
    its1, res1, T1 = run(op, model, seed=99)
    gain = [r0 / r1 for r0, r1 in zip(res0[1:], res1[1:])]
    print("initial residual gain per step", [round(x, 2) for x in gain],
          "iterations", sum(its0), "->", sum(its1))
    # the step-length scaling makes the guess's residual never exceed the extrapolation's
    assert all(r1 <= r0 * 1.0001 for r0, r1 in zip(res0[1:], res1[1:]))
    assert max(gain) > 1.5  # the network removes a real part of the extrapolation error
    # measured on this pool: 1.1-2.1x smaller initial residual but no fewer CG iterations
    # (132 -> 134); the solver iterates to the same tolerance, so at most a few more
    assert sum(its1) <= 1.05 * sum(its0) + 1
    # both runs stop at |b - J T| <= 1e-8 |b| from different guesses, so the fields may
    # differ by up to ~cond(J) * 1e-8 per step (measured 6e-6 after 14 steps)
    assert torch.linalg.vector_norm(T1 - T0) <= 5e-5 * torch.linalg.vector_norm(T0)


def test_guess_rejects_a_network_of_another_grid():
    op = LG.make_operator(8)  # 25^3 nodal grid
    model = LG.GuessModel(stride=1, T_scale=0.1, net=LG.UNet((17, 17, 17)))
    T = op.new_vector()
    with pytest.raises(H.ExcInvalidArgument):
        model.guess(op, T, T, None, LG.DT)


def test_learned_direction_starts_the_increment_solve_closer():
    """PREDICTOR_LINEAR_DIRECTION: linearised at the extrapolation (as PREDICTOR_LINEAR), the
    increment solve starts from alpha d with alpha minimising the residual, so the initial
    residual never exceeds the extrapolation's and the converged fields are the same to the
    solver tolerance (the linearisation point is the same; only the start differs)."""
    op = LG.make_operator(32)
    model = LG.GuessModel.load(MODEL, stride=1)
    its0, res0, T0 = run(op, None, seed=77, n_steps=8)
    its1, res1, T1 = run(op, model, seed=77, n_steps=8, direction=True)
    print("initial residual", [f"{a:.2e}->{b:.2e}" for a, b in zip(res0, res1)],
          "iterations", sum(its0), "->", sum(its1))
    assert all(r1 <= r0 * (1 + 1e-9) for r0, r1 in zip(res0, res1))
    assert any(r1 < 0.9 * r0 for r0, r1 in zip(res0[1:], res1[1:]))
    # same linearisation points, different starts: the fields differ by the solver tolerance
    assert torch.linalg.vector_norm(T1 - T0) <= 2e-5 * torch.linalg.vector_norm(T0)


def test_direction_predictor_needs_a_direction_and_one_linearisation():
    op = LG.make_operator(4)
    opn = H.HeatDiffuseOperation(op, H.LinearSolverData(), predictor=L.PREDICTOR_LINEAR_DIRECTION,
                                 single_linearization=True)
    with pytest.raises(H.ExcInvalidArgument):
        opn.solve(LG.DT)
    opn.set_direction(op.new_vector())
    opn.params.single_linearization = 0
    with pytest.raises(H.ExcInvalidArgument):
        opn.solve(LG.DT)
    opn.params.single_linearization = 1
    st = opn.solve(LG.DT)  # a zero direction: the plain linear-predictor step
    assert st.converged == 1


def test_streaming_training_and_held_out_evaluation_run(tmp_path):
    """The streaming trainer (samples consumed as the solver produces them) and the held-out
    evaluation on a small mesh: losses are finite, every trajectory after its first step gives a
    sample, and the evaluation reports iterations and times for both predictors."""
    op = LG.make_operator(8)
    net = LG.UNet(op.dims, seed=3)
    hist, seen, done = LG.train_streaming(op, net, n_traj=2, n_steps=4, seed=5, passes=2)
    assert done == 2 and seen == 2 * 3 and len(hist) == 2 * seen
    assert all(h == h and h < 1e6 for h in hist)
    model = LG.GuessModel(stride=1, T_scale=0.1, net=net)
    model.save(str(tmp_path / "m"))
    ev = LG.evaluate(op, LG.GuessModel.load(str(tmp_path / "m")), seeds=[7], n_steps=3)
    for name in ("extrapolation", "learned"):
        assert len(ev[name]["iterations"]) == 2 and ev[name]["mean_ms"] > 0.0
