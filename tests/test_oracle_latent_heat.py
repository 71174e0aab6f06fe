"""Latent heat of fusion as an apparent heat capacity in the mushy zone (oracle), pinned by the
properties the reference's unit test checks (unit_tests/heat/apparent_capacity.cpp: L = 338e3,
T_solidus 271, T_liquidus 275): zero value and slope at the mushy-zone bounds for poly4_bell,
the integral over the mushy zone equal to the latent heat, the temperature derivative against
central differences; and the heat tangent with it is the derivative of the residual."""
import numpy as np
import pytest

from oracle import oracle as O

TYPES = {"poly4_bell": (O.APPARENT_POLY4_BELL, True), "constant": (O.APPARENT_CONSTANT, False),
         "qlq": (O.APPARENT_QLQ, False)}
L, TS, TL = 338e3, 271.0, 275.0


def capacity(kind):
    """A(T) and dA/dT: rho = 1 and cp = 0 in both phases leave rho*cp = A."""
    m = O.material(O.LAW_LIQUID_SOLID, rho=1.0, cp=0.0, k=1.0, T_solidus=TS, T_liquidus=TL,
                   latent_heat=L, apparent_capacity=TYPES[kind][0])
    return (lambda T: O.material_eval(m, T)[0]), (lambda T: O.material_eval(m, T)[2])


@pytest.mark.parametrize("kind", list(TYPES))
def test_zero_at_solidus_and_liquidus(kind):
    if not TYPES[kind][1]:
        pytest.skip("this profile is not expected to vanish at the mushy-zone bounds")
    A, dA = capacity(kind)
    for T in (TS, TL):
        assert abs(A(T)) < 1e-6 and abs(dA(T)) < 1e-6


@pytest.mark.parametrize("kind", list(TYPES))
def test_integral_equals_latent_heat(kind):
    A, _ = capacity(kind)
    n = 1000
    h = (TL - TS) / n
    integral = h * sum(A(TS + (i + 0.5) * h) for i in range(n))
    assert abs(integral - L) / L < 1e-8


@pytest.mark.parametrize("kind", list(TYPES))
def test_temperature_derivative_matches_finite_differences(kind):
    A, dA = capacity(kind)
    eps = 1e-5
    for i in range(3):
        T = TS + 0.1 + i * (TL - TS) / 5.0
        expected = (A(T + eps) - A(T - eps)) / (2.0 * eps)
        assert abs(dA(T) - expected) <= 1e-5 * max(1.0, abs(expected)), T


def test_outside_the_mushy_zone_and_without_latent_heat_nothing_changes():
    base = O.material(O.LAW_LIQUID_SOLID, rho=1000.0, cp=4226.0, k=0.556, rho_s=900.0,
                      cp_s=1762.0, k_s=2.22, T_solidus=TS, T_liquidus=TL)
    lat = O.material(O.LAW_LIQUID_SOLID, rho=1000.0, cp=4226.0, k=0.556, rho_s=900.0,
                     cp_s=1762.0, k_s=2.22, T_solidus=TS, T_liquidus=TL, latent_heat=L)
    for T in (250.0, TS, TL, 300.0):
        assert O.material_eval(lat, T) == O.material_eval(base, T)
    a, b = O.material_eval(lat, 273.0), O.material_eval(base, 273.0)
    assert a[1] == b[1] and a[0] > b[0]  # conductivity unchanged, capacity raised


@pytest.mark.parametrize("kind", ["poly4_bell", "qlq"])
def test_tangent_with_latent_heat_is_derivative_of_residual(kind):
    """d(rho_cp)/dT (T - T_old)/dt u with the apparent capacity's slope in the tangent
    (heat_diffuse_operator.cpp:1046-1047) is the derivative of the residual; both forms agree."""
    rng = np.random.default_rng(12)
    o = O.Oracle(2, (3, 3, 3), perturb=0.1, seed=4)
    o.set_material(O.material(O.LAW_LIQUID_SOLID, rho=1000.0, cp=4226.0, k=0.556, rho_s=900.0,
                              cp_s=1762.0, k_s=2.22, T_solidus=0.2, T_liquidus=0.8,
                              latent_heat=5e3, apparent_capacity=TYPES[kind][0]), 1e-2)
    T = rng.uniform(0, 1, o.n_dofs)
    T_old = rng.uniform(0, 1, o.n_dofs)
    du = rng.uniform(-1, 1, o.n_dofs)
    du[o.mask().astype(bool)] = 0.0
    eps = 1e-6
    fd = -(o.create_rhs(T + eps * du, T_old) - o.create_rhs(T - eps * du, T_old)) / (2 * eps)
    Jdu = o.vmult(du, T, T_old)
    assert np.abs(fd - Jdu).max() <= 1e-6 * np.abs(Jdu).max()
    assert np.abs(Jdu - o.vmult(du, T, T_old, form=1)).max() <= 1e-13 * np.abs(Jdu).max()


def test_volume_specific_capacity_with_latent_heat_is_rejected():
    o = O.Oracle(1, (2, 2, 2))
    with pytest.raises(ValueError):
        o.set_material(O.material(O.LAW_LIQUID_SOLID, volume_specific=True, T_solidus=0.2,
                                  T_liquidus=0.8, latent_heat=1.0), 1e-2)


# the product's law, evaluated on the host by the code the cell kernels run, against the oracle
PRODUCT_CASES = [
    ("liquid_solid", dict(law=2), False),
    ("liquid_solid_sharp", dict(law=2, sharp=True), False),
    ("three_phase", dict(law=4), True),
    ("three_phase_sharp_gl", dict(law=4, sharp_gas_liquid=True), True),
]


@pytest.mark.parametrize("name,kw,uses_h", PRODUCT_CASES)
@pytest.mark.parametrize("kind", list(TYPES) + ["none"])
def test_product_material_law_matches_oracle(name, kw, uses_h, kind):
    from meltpooldg_b200 import heat as H
    props = dict(rho=7850.0, cp=460.0, k=55.563, rho_s=7000.0, cp_s=700.0, k_s=30.0,
                 T_solidus=TS, T_liquidus=TL, rho_g=1.2, cp_g=1000.0, k_g=0.03)
    latent, prof = (0.0, 0) if kind == "none" else (L, TYPES[kind][0])
    om = O.material(latent_heat=latent, apparent_capacity=prof, **props, **kw)
    pm = H.material(**props, **kw)
    for T in np.linspace(265.0, 281.0, 41):
        for Hv in ((0.0, 0.3, 0.6, 1.0) if uses_h else (1.0,)):
            a = np.array(O.material_eval(om, T, Hv))
            b = np.array(H.material_eval(pm, T, Hv, latent, prof))
            assert np.allclose(b, a, rtol=1e-13, atol=1e-9), (T, Hv, a, b)


def test_product_rejects_latent_heat_with_volume_specific_capacity():
    from meltpooldg_b200 import heat as H
    pm = H.material(law=2, T_solidus=TS, T_liquidus=TL, volume_specific=True)
    with pytest.raises(H.ExcNotImplemented):
        H.material_eval(pm, 273.0, 1.0, L, 0)
    assert H.material_eval(pm, 273.0, 1.0, 0.0, 0)[0] > 0.0
