"""The laser's motion and power over time (meltpooldg_b200.laser, host logic, no GPU): the
semantics of source/heat/laser_operation.cpp:229-320 on hand-computed cases, and the arguments
it hands to the operator's source kernels."""
import math

import pytest

from meltpooldg_b200 import _lib as L
from meltpooldg_b200.heat import ExcInvalidArgument, ExcNotImplemented
from meltpooldg_b200.laser import LaserData, LaserOperation


class FakeOperator:
    def __init__(self):
        self.calls = []

    def laser_source(self, q, profile, **kw):
        self.calls.append(("laser_source", profile, kw))
        return q

    def set_laser(self, profile=None, **kw):
        self.calls.append(("set_laser", profile, kw))


def test_moves_along_the_normalised_scan_direction():
    las = LaserOperation(LaserData(power=100.0, scan_speed=0.5, starting_position=(0.1, 0.2, 0.3),
                                   scan_direction=(3.0, 0.0, 4.0)))
    las.reset(0.0)
    assert las.get_laser_position() == (0.1, 0.2, 0.3) and las.get_laser_power() == 100.0
    for _ in range(4):
        assert las.move_laser(0.1)
    x, y, z = las.get_laser_position()
    assert math.isclose(x, 0.1 + 0.6 * 0.2) and y == 0.2 and math.isclose(z, 0.3 + 0.8 * 0.2)
    assert math.isclose(las.current_time, 0.4)


def test_static_beam_reports_no_change_while_the_power_is_constant():
    las = LaserOperation(LaserData(power=5.0))
    las.reset(0.0)
    assert not las.move_laser(1e-3)
    assert las.get_laser_position() == (0.0, 0.0, 0.0) and las.get_laser_power() == 5.0


def test_constant_power_switches_off_at_the_end_time():
    las = LaserOperation(LaserData(power=10.0, power_end_time=0.25))
    las.reset(0.0)
    assert not las.move_laser(0.1)   # t = 0.1
    assert not las.move_laser(0.1)   # t = 0.2
    assert las.move_laser(0.1)       # t = 0.3 >= 0.25: off
    assert las.get_laser_power() == 0.0
    las.reset(0.0)                   # back on, beam at its start
    assert las.get_laser_power() == 10.0


def test_ramp_is_linear_and_clamped():
    las = LaserOperation(LaserData(power=8.0, power_over_time="ramp", power_start_time=0.1,
                                   power_end_time=0.5, scan_speed=1.0))
    las.reset(0.0)
    assert las.get_laser_power() == 0.0
    powers = []
    for _ in range(7):
        las.move_laser(0.1)
        powers.append(las.get_laser_power())
    assert [round(p, 12) for p in powers] == [0.0, 2.0, 4.0, 6.0, 8.0, 8.0, 8.0]


def test_invalid_parameters_are_rejected():
    with pytest.raises(ExcInvalidArgument):
        LaserOperation(LaserData(power_start_time=1.0, power_end_time=1.0))
    with pytest.raises(ExcNotImplemented):
        LaserOperation(LaserData(power_over_time="pulsed"))
    with pytest.raises(ExcInvalidArgument):
        LaserOperation(LaserData(scan_direction=(0.0, 0.0, 0.0)))


def test_hands_the_current_beam_to_the_source_kernels():
    op = FakeOperator()
    las = LaserOperation(LaserData(intensity_profile=L.LASER_GUSAROV, power=3.0, radius=0.1,
                                   scan_speed=2.0, gusarov=(0.7, 6e4, 5e-5),
                                   beam_direction=(0.0, 0.0, -2.0)), op)
    las.reset(0.0)
    las.move_laser(0.5)
    las.compute_heat_source("q")
    las.attach()
    las.detach()
    (n0, p0, k0), (n1, p1, k1), (n2, p2, k2) = op.calls
    assert n0 == "laser_source" and n1 == "set_laser" and p0 == p1 == L.LASER_GUSAROV
    assert k0 == k1 and k0["power"] == 3.0 and k0["position"] == (1.0, 0.0, 0.0)
    assert k0["direction"] == (0.0, 0.0, -1.0) and k0["gusarov"] == (0.7, 6e4, 5e-5)
    assert n2 == "set_laser" and p2 is None
