"""The laser's motion and power over time, driving the device source kernels.

Mirrors MeltPoolDG's `LaserOperation` for the volumetric models (source/heat/laser_operation.cpp):
`reset(start_time)` (:229-240) puts the beam at its starting position and evaluates the power at
the start time; `move_laser(dt)` (:245-270) advances the time, moves the beam by
`scan_direction / |scan_direction| * scan_speed * dt` when the scan speed is non-zero and
re-evaluates the power; `compute_laser_intensity()` (:296-320) is the "ramp" (linear from
`power_start_time` to `power_end_time`, clamped to [0, 1]) or "constant" (1 before
`power_end_time`, 0 from it on) factor of the nominal power. The source itself is evaluated on
the device: `compute_heat_source(q)` writes the profile at the support points
(`LaserHeatSourceVolumetric::compute_volumetric_heat_source`, laser_heat_source_volumetric.cpp:
20-58) and `attach()` hands the current beam to the operator so that the residual kernels
evaluate it in place of a nodal source (`mpdg_heat_set_laser`)."""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence

from . import _lib as L
from .heat import ExcInvalidArgument, ExcNotImplemented


@dataclass
class LaserData:
    """`LaserData` (include/meltpooldg/heat/laser_data.hpp:47-97) for the volumetric models."""
    intensity_profile: int = L.LASER_GAUSS_VOLUMETRIC
    power: float = 0.0
    power_over_time: str = "constant"
    power_start_time: float = 0.0
    power_end_time: float = math.inf
    scan_speed: float = 0.0
    starting_position: Sequence[float] = (0.0, 0.0, 0.0)
    scan_direction: Sequence[float] = (1.0, 0.0, 0.0)
    beam_direction: Sequence[float] = (0.0, 0.0, -1.0)
    radius: float = 0.0
    gusarov: Sequence[float] = (0.0, 0.0, 0.0)  # reflectivity, extinction coefficient, layer
    planar: bool = False  # 2D profile in the x-z plane (mesh one cell thick in y)


def _unit(v: Sequence[float]):
    n = math.sqrt(sum(float(c) * float(c) for c in v))
    if n == 0.0:
        raise ExcInvalidArgument("laser direction of zero length")
    return tuple(float(c) / n for c in v)


class LaserOperation:
    def __init__(self, data: LaserData, operator=None):
        if not data.power_end_time > data.power_start_time:
            raise ExcInvalidArgument(
                "For the temporal ramp distribution of the laser power, the parameter laser "
                "power end time must be larger than laser power start time.")
        if data.power_over_time not in ("ramp", "constant"):
            raise ExcNotImplemented(f"power over time '{data.power_over_time}'")
        self.data = data
        self.op = operator
        self.scan_direction = _unit(data.scan_direction)
        self.beam_direction = _unit(data.beam_direction)
        self.current_time = 0.0
        self.laser_intensity = math.nan  # set by reset()
        self.current_power = 0.0
        self.laser_position = tuple(float(c) for c in data.starting_position)

    def reset(self, start_time: float = 0.0):
        self.current_time = float(start_time)
        self.compute_laser_intensity()
        self.laser_position = tuple(float(c) for c in self.data.starting_position)

    def compute_laser_intensity(self) -> bool:
        """The power factor at the current time; True when it changed."""
        previous = self.laser_intensity
        d = self.data
        if d.power_over_time == "ramp":
            s = (self.current_time - d.power_start_time) / (d.power_end_time - d.power_start_time)
            self.laser_intensity = min(max(0.0, s), 1.0)
        else:
            self.laser_intensity = 0.0 if self.current_time >= d.power_end_time else 1.0
        self.current_power = d.power * self.laser_intensity
        return previous != self.laser_intensity

    def move_laser(self, dt: float) -> bool:
        """Advance by dt; True when the position or the power changed."""
        changed = False
        self.current_time += float(dt)
        if self.data.scan_speed != 0.0:
            s = self.data.scan_speed * float(dt)
            self.laser_position = tuple(p + s * e for p, e in
                                        zip(self.laser_position, self.scan_direction))
            changed = True
        return self.compute_laser_intensity() or changed

    def get_laser_position(self):
        return self.laser_position

    def get_laser_power(self) -> float:
        return self.current_power

    def _args(self):
        d = self.data
        return dict(power=self.current_power, position=self.laser_position, radius=d.radius,
                    direction=self.beam_direction, gusarov=tuple(d.gusarov), planar=d.planar)

    def compute_heat_source(self, q, operator=None):
        """q = the intensity profile at the support points (the device kernel)."""
        op = operator or self.op
        if op is None:
            raise ExcInvalidArgument("no operator to evaluate the laser on")
        return op.laser_source(q, self.data.intensity_profile, **self._args())

    def attach(self, operator=None):
        """The current beam as the residual's source (evaluated in the create_rhs kernels
        wherever the heat source is None); call after every move_laser."""
        op = operator or self.op
        if op is None:
            raise ExcInvalidArgument("no operator to attach the laser to")
        op.set_laser(self.data.intensity_profile, **self._args())

    def detach(self, operator=None):
        (operator or self.op).set_laser(None)


__all__ = ["LaserData", "LaserOperation"]
