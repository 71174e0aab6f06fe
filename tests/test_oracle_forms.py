"""The oracle's two independent forms agree (sum factorisation vs direct quadrature)."""
import numpy as np
import pytest

from oracle import oracle as O

LAWS = {
    "constant": O.material(),
    "linear_k": O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5),
    "liquid_solid": O.material(O.LAW_LIQUID_SOLID, rho=1000.0, cp=4226.0, k=0.556, rho_s=900.0,
                               cp_s=1762.0, k_s=2.22, T_solidus=0.2, T_liquidus=0.8),
}


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("perturb", [0.0, 0.2])
@pytest.mark.parametrize("law", list(LAWS))
def test_sum_factorisation_matches_direct_quadrature(degree, perturb, law):
    rng = np.random.default_rng(degree)
    o = O.Oracle(degree, (3, 2, 3), perturb=perturb, seed=11)
    o.set_material(LAWS[law], 1e-3)
    src = rng.uniform(-1, 1, o.n_dofs)
    T_lin = rng.uniform(0, 1, o.n_dofs)
    T_old = rng.uniform(0, 1, o.n_dofs)
    a = o.vmult(src, T_lin, T_old, form=0)
    b = o.vmult(src, T_lin, T_old, form=1)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    da = o.inverse_diagonal(T_lin, T_old, form=0)
    db = o.inverse_diagonal(T_lin, T_old, form=1)
    assert np.allclose(1 / da, 1 / db, rtol=1e-12, atol=0)
    # constrained rows of vmult are zero, inverse diagonal there is one
    m = o.mask().astype(bool)
    assert np.all(a[m] == 0.0) and np.all(da[m] == 1.0)


def test_operator_symmetric_for_constant_law():
    rng = np.random.default_rng(3)
    o = O.Oracle(3, (3, 3, 3), perturb=0.2, seed=2)
    o.set_material(LAWS["constant"], 1e-3)
    u = rng.uniform(-1, 1, o.n_dofs)
    v = rng.uniform(-1, 1, o.n_dofs)
    assert abs(u @ o.vmult(v) - v @ o.vmult(u)) <= 1e-12 * abs(u @ o.vmult(u))


def test_tangent_is_derivative_of_residual():
    """J(T) du = d/deps [-R(T + eps du)] * (-1): the tangent of the k(T) law is consistent."""
    rng = np.random.default_rng(5)
    o = O.Oracle(2, (3, 3, 3), perturb=0.1, seed=4)
    o.set_material(LAWS["linear_k"], 1e-2)
    T = rng.uniform(0, 1, o.n_dofs)
    T_old = rng.uniform(0, 1, o.n_dofs)
    du = rng.uniform(-1, 1, o.n_dofs)
    du[o.mask().astype(bool)] = 0.0
    eps = 1e-6
    rp = o.create_rhs(T + eps * du, T_old)
    rm = o.create_rhs(T - eps * du, T_old)
    fd = -(rp - rm) / (2 * eps)
    Jdu = o.vmult(du, T, T_old)
    assert np.abs(fd - Jdu).max() <= 1e-7 * np.abs(Jdu).max()


def test_boundary_tangent_is_derivative_of_boundary_residual():
    rng = np.random.default_rng(8)
    o = O.Oracle(2, (3, 3, 3), perturb=0.15, seed=1, dirichlet_mask=0b001100)
    o.set_material(LAWS["constant"], 1e-2)
    o.set_boundary(0, convection=(5.0, 300.0), radiation=(0.8, 320.0))
    o.set_boundary(5, radiation=(0.5, 250.0))
    o.set_boundary(1, neumann=3.0)
    T = rng.uniform(900, 1100, o.n_dofs)
    T_old = rng.uniform(900, 1100, o.n_dofs)
    du = rng.uniform(-1, 1, o.n_dofs)
    du[o.mask().astype(bool)] = 0.0
    eps = 1e-3
    fd = -(o.create_rhs(T + eps * du, T_old) - o.create_rhs(T - eps * du, T_old)) / (2 * eps)
    Jdu = o.vmult(du, T, T_old)
    assert np.abs(fd - Jdu).max() <= 1e-7 * np.abs(Jdu).max()
    # the boundary terms are in the diagonal too
    d0 = 1.0 / o.inverse_diagonal(T, T_old, form=0)
    d1 = 1.0 / o.inverse_diagonal(T, T_old, form=1)
    assert np.allclose(d0, d1, rtol=1e-12, atol=0)


def test_picard_forms_reduce_to_the_constant_law():
    """The Picard operator (form 2) and its diagonal at a constant linearisation point
    T = c equal the constant-conductivity operator with k = k0 + k1 c."""
    import numpy as np
    from oracle import oracle as O
    o = O.Oracle(3, (3, 2, 3), perturb=0.2, seed=3)
    o.set_material(O.material(O.LAW_LINEAR_K, k=1.0, k1=0.5), 1e-3)
    c = O.Oracle(3, (3, 2, 3), perturb=0.2, seed=3)
    c.set_material(O.material(O.LAW_CONSTANT, k=1.4), 1e-3)
    rng = np.random.default_rng(0)
    src = rng.uniform(-1, 1, o.n_dofs)
    T = np.full(o.n_dofs, 0.8)
    a, b = o.vmult(src, T, T, form=2), c.vmult(src)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    da, db = o.inverse_diagonal(T, T, form=2), c.inverse_diagonal()
    assert np.abs(da - db).max() <= 1e-13 * np.abs(db).max()
    # away from a constant point the Picard diagonal differs from the tangent's
    T2 = rng.uniform(0.0, 1.0, o.n_dofs)
    assert np.abs(o.inverse_diagonal(T2, T2, form=2) - o.inverse_diagonal(T2, T2)).max() > 0


def test_laser_profiles_follow_their_formulas():
    """Volumetric laser intensity at the support points: the uniform profile is the power,
    the Gauss profiles peak at power / (r sqrt(pi/2))^3 (volumetric) and power / (r^2 pi/2)
    (projection, constant along the beam), the Gusarov profile vanishes outside the layer."""
    import math

    import numpy as np
    from oracle import oracle as O
    o = O.Oracle(2, (4, 4, 4), perturb=0.1, seed=1)
    x = o.support_points()
    P, r, c = 30.0, 0.3, np.array([0.5, 0.5, 1.0])
    assert np.all(o.laser_source(0, P, c) == P)
    qv = o.laser_source(1, P, c, radius=r)
    d2 = ((x - c) ** 2).sum(1)
    ref = P / (r * math.sqrt(math.pi / 2)) ** 3 * np.exp(-2 * d2 / r ** 2)
    assert np.abs(qv - ref).max() <= 1e-13 * ref.max()
    qp = o.laser_source(2, P, c, radius=r, direction=(0.0, 0.0, -1.0))
    dl2 = ((x[:, :2] - c[:2]) ** 2).sum(1)
    ref = P / (r * r * math.pi / 2) * np.exp(-2 * dl2 / r ** 2)
    assert np.abs(qp - ref).max() <= 1e-13 * ref.max()
    # Gusarov: powder surface z = 0 with the material below (the reference's convention;
    # its "z < position_z" compares the depth with the centre height), layer L = 0.5
    b = O.Oracle(2, (4, 4, 4), lo=(0, 0, -1), hi=(1, 1, 0), perturb=0.1, seed=1)
    xb = b.support_points()
    g = b.laser_source(3, P, (0.5, 0.5, 0.0), radius=0.6, gusarov=(0.6, 20.0, 0.5))
    depth = -xb[:, 2]
    dist = np.sqrt(((xb - np.array([0.5, 0.5, 0.0])) ** 2).sum(1))
    outside = (depth >= 0.5) | (depth < 0.0) | (dist > 0.6)
    assert np.all(g[outside] == 0.0) and np.all(np.isfinite(g))
    assert np.abs(g[~outside]).max() > 0.0


GAS_LIQUID = dict(rho=2.0, cp=3.0, k=5.0, rho_g=0.5, cp_g=1.5, k_g=0.3)


def transport_fields(o, velocity=True):
    x = o.support_points()
    H = 0.5 + 0.5 * np.tanh((x[:, 0] - 0.45) / 0.1)
    V = np.stack([np.sin(3 * x[:, 1]), 0.5 + x[:, 2], -x[:, 0] * x[:, 1]]) if velocity else None
    return H, V


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("perturb", [0.0, 0.2])
@pytest.mark.parametrize("sharp,vs", [(False, False), (True, False), (False, True)])
def test_two_phase_transport_forms_agree(degree, perturb, sharp, vs):
    """Gas-liquid law on a heaviside field plus convection: both forms agree, the
    residual is the affine counterpart of the tangent (the law is linear in T) and the
    Picard form equals the tangent (no temperature derivatives)."""
    o = O.Oracle(degree, (3, 2, 3), perturb=perturb, seed=7, hi=(1.0, 1.3, 0.8))
    o.set_material(O.material(O.LAW_GAS_LIQUID, sharp_gas_liquid=sharp, volume_specific=vs,
                              **GAS_LIQUID), 1e-2)
    o.set_fields(*transport_fields(o))
    rng = np.random.default_rng(degree)
    u = rng.standard_normal(o.n_dofs)
    a = o.vmult(u, form=0)
    assert np.abs(a - o.vmult(u, form=1)).max() <= 1e-13 * np.abs(a).max()
    assert np.array_equal(a, o.vmult(u, form=2))
    da, db = o.inverse_diagonal(form=0), o.inverse_diagonal(form=1)
    assert np.allclose(1 / da, 1 / db, rtol=1e-12, atol=0)
    T, To = rng.standard_normal(o.n_dofs), rng.standard_normal(o.n_dofs)
    u[o.mask().astype(bool)] = 0.0
    lin = o.create_rhs(T, To) - o.create_rhs(T + u, To)
    assert np.abs(lin - o.vmult(u)).max() <= 1e-12 * np.abs(lin).max()


def test_diagonal_of_the_convective_operator_matches_its_columns():
    o = O.Oracle(2, (2, 2, 2), perturb=0.2, seed=4)
    o.set_material(O.material(O.LAW_GAS_LIQUID, **GAS_LIQUID), 1e-2)
    o.set_fields(*transport_fields(o))
    N = o.n_dofs
    m = o.mask().astype(bool)
    col = np.array([o.vmult(np.eye(N)[i])[i] for i in range(N)])
    inv = o.inverse_diagonal()
    assert np.allclose(inv[~m], 1 / col[~m], rtol=1e-13, atol=0) and np.all(inv[m] == 1.0)


def test_convection_of_a_linear_field():
    """Constant velocity v and T = a.x with T_old = T: the interior residual rows are
    -rho_cp (v.a) int(phi_i) (the diffusive part integrates to zero there)."""
    for degree, perturb in [(2, 0.2), (3, 0.15)]:
        o = O.Oracle(degree, (3, 4, 3), perturb=perturb)
        x = o.support_points()
        a, v = np.array([0.7, -1.1, 0.4]), np.array([1.0, 2.0, -3.0])
        T = x @ a
        o.set_material(O.material(rho=2.0, cp=3.0, k=5.0), 1e-2)
        o.set_fields(None, np.tile(v[:, None], (1, o.n_dofs)))
        r = o.create_rhs(T, T)
        o.set_fields(None, None)
        int_phi = o.create_rhs(0 * T, 0 * T, heat_source=np.ones(o.n_dofs))
        inner = o.mask() == 0
        assert np.abs(r[inner] + 6.0 * (v @ a) * int_phi[inner]).max() <= 1e-13 * np.abs(r).max()


@pytest.mark.parametrize("sharp,vs", [(False, False), (True, False), (False, True), (True, True)])
def test_uniform_heaviside_mixes_the_phase_properties(sharp, vs):
    """A uniform heaviside H = 0.3 gives the constant law with the mixed properties
    (1 - w) gas + w liquid, w = H or H > 0.5 (material.templates.hpp:240-295, :515-524)."""
    g = GAS_LIQUID
    o = O.Oracle(2, (3, 3, 2), perturb=0.1, seed=3)
    u = np.random.default_rng(0).standard_normal(o.n_dofs)
    o.set_material(O.material(O.LAW_GAS_LIQUID, sharp_gas_liquid=sharp, volume_specific=vs, **g),
                   1e-2)
    o.set_fields(np.full(o.n_dofs, 0.3), None)
    a = o.vmult(u)
    w = 0.0 if sharp else 0.3
    mix = lambda liq, gas: (1 - w) * gas + w * liq
    k = mix(g["k"], g["k_g"])
    rhocp = mix(g["rho"] * g["cp"], g["rho_g"] * g["cp_g"]) if vs else \
        mix(g["rho"], g["rho_g"]) * mix(g["cp"], g["cp_g"])
    o.set_fields(None, None)
    o.set_material(O.material(rho=rhocp, cp=1.0, k=k), 1e-2)
    assert np.abs(a - o.vmult(u)).max() <= 1e-13 * np.abs(a).max()


def test_velocity_needs_a_temperature_independent_law():
    o = O.Oracle(1, (2, 2, 2))
    o.set_material(O.material(O.LAW_LINEAR_K, k1=0.5), 1e-2)
    with pytest.raises(ValueError):
        o.set_fields(None, np.zeros((3, o.n_dofs)))


THREE_PHASE = dict(rho=1.0, cp=1.0, k=0.5, rho_s=1.2, cp_s=0.8, k_s=2.5, T_solidus=0.3,
                   T_liquidus=0.7, rho_g=0.4, cp_g=1.5, k_g=0.2)


@pytest.mark.parametrize("law,sharp_gl,vs", [(O.LAW_LIQUID_SOLID, False, False),
                                             (O.LAW_LIQUID_SOLID, False, True),
                                             (O.LAW_GAS_LIQUID_SOLID, False, False),
                                             (O.LAW_GAS_LIQUID_SOLID, True, False),
                                             (O.LAW_GAS_LIQUID_SOLID, False, True)])
def test_transport_tangent_is_derivative_of_residual(law, sharp_gl, vs):
    """Temperature-dependent laws with a velocity (and the three-phase law on a heaviside):
    the tangent, including d(rho_cp)/dT (v.grad T) u (heat_diffuse_operator.cpp:1044-1049),
    is the derivative of the residual; both forms and the diagonal agree."""
    rng = np.random.default_rng(9)
    o = O.Oracle(2, (3, 3, 3), perturb=0.1, seed=4)
    o.set_material(O.material(law, sharp_gas_liquid=sharp_gl, volume_specific=vs, **THREE_PHASE),
                   1e-2)
    Hf, V = transport_fields(o)
    o.set_fields(Hf if law == O.LAW_GAS_LIQUID_SOLID else None, V)
    T = rng.uniform(0, 1, o.n_dofs)
    T_old = rng.uniform(0, 1, o.n_dofs)
    du = rng.uniform(-1, 1, o.n_dofs)
    du[o.mask().astype(bool)] = 0.0
    eps = 1e-6
    fd = -(o.create_rhs(T + eps * du, T_old) - o.create_rhs(T - eps * du, T_old)) / (2 * eps)
    Jdu = o.vmult(du, T, T_old)
    assert np.abs(fd - Jdu).max() <= 1e-6 * np.abs(Jdu).max()
    assert np.abs(Jdu - o.vmult(du, T, T_old, form=1)).max() <= 1e-13 * np.abs(Jdu).max()
    da, db = o.inverse_diagonal(T, T_old, form=0), o.inverse_diagonal(T, T_old, form=1)
    assert np.allclose(1 / da, 1 / db, rtol=1e-12, atol=0)


def test_three_phase_law_limits():
    """H = 1 gives the liquid-solid law, H = 0 the gas (constant) law."""
    o = O.Oracle(2, (3, 2, 2), perturb=0.1, seed=3)
    rng = np.random.default_rng(1)
    u, T, To = (rng.uniform(-1, 1, o.n_dofs), rng.uniform(0, 1, o.n_dofs),
                rng.uniform(0, 1, o.n_dofs))
    def op(m, H):
        o.set_fields(None, None)
        o.set_material(m, 1e-2)
        o.set_fields(H, None)
        return o.vmult(u, T, To), o.create_rhs(T, To)
    three = O.material(O.LAW_GAS_LIQUID_SOLID, **THREE_PHASE)
    a = op(three, np.ones(o.n_dofs))
    b = op(O.material(O.LAW_LIQUID_SOLID, **THREE_PHASE), None)
    assert all(np.abs(x - y).max() <= 1e-14 * np.abs(y).max() for x, y in zip(a, b))
    a = op(three, np.zeros(o.n_dofs))
    g = THREE_PHASE
    b = op(O.material(rho=g["rho_g"], cp=g["cp_g"], k=g["k_g"]), None)
    assert all(np.abs(x - y).max() <= 1e-14 * np.abs(y).max() for x, y in zip(a, b))
