"""Channel cross-section and the 1D Manning discharge that feeds a 3D reach.

``Section`` has the fields and meaning of the reference's compound section
(floodsim/geometry.py:25-38): a trapezoidal main channel of bottom width B, bank
height Hb and side slope z (horizontal : vertical), flanked by floodplains of
width Bf per side; n and nf are the Manning coefficients of channel and
floodplain.  ``manning_discharge`` gives the uniform-flow discharge of the
in-bank trapezoid, Q = A R^(2/3) sqrt(S) / n (floodsim/hydraulics1d.py:26-53
for h <= Hb), which is how the large single-case workload sets its inflow.
"""
from __future__ import annotations

import math
from dataclasses import dataclass


@dataclass
class Section:
    B: float = 40.0      # channel bottom width (m)
    Hb: float = 3.0      # bank height (m)
    z: float = 2.0       # bank slope, horizontal per vertical
    Bf: float = 200.0    # floodplain width per side (m)
    n: float = 0.032     # Manning n of the channel
    nf: float = 0.06     # Manning n of the floodplains

    @property
    def Tb(self) -> float:
        """Width at bank-full stage."""
        return self.B + 2 * self.z * self.Hb


def manning_discharge(sec: Section, h: float, slope: float) -> float:
    """Uniform-flow discharge (m^3/s) of the trapezoidal channel at depth h <= Hb."""
    if h > sec.Hb:
        raise ValueError("manning_discharge covers in-bank stages (h <= Hb)")
    area = (sec.B + sec.z * h) * h
    wetted = sec.B + 2.0 * h * math.sqrt(1.0 + sec.z * sec.z)
    radius = area / wetted
    return area * radius ** (2.0 / 3.0) * math.sqrt(slope) / sec.n
