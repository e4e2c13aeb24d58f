"""Seeded boat cases of the benchmark workloads.

* ``config1_case`` -- 48 m x 12 m x 3 m rectangular channel at dx = 0.25 m, Manning
  n = 0.03, mean inflow 0.8 m/s, Smagorinsky Cs = 0.12, one 10 m x 2 m x 0.8 m long-tail-
  style boat centred 16 m downstream with one 0.30 m / 75 kW propeller 0.35 m deep, tilted
  12 deg down.  The reference's grid rule gives 192 x 50 x 12 cells.
* ``config2_case`` -- 150 m trapezoidal reach, 60 m top width, 1:2 banks, 4 m deep,
  dx = 0.1 m (1500 x 602 x 40 = 36.1M cells), Manning n = 0.025, inflow the uniform-flow
  discharge at the 4 m stage (bed slope 3e-4), bed perturbed by a seeded Gaussian random
  field (sigma 0.15 m, correlation length 5 m), one 20 m x 6 m x 1.5 m pusher tug with two
  1.2 m / 300 kW propellers under the stern.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
from scipy.ndimage import gaussian_filter

from .geometry import Section, manning_discharge
from .reach3d import BoatType, Fleet, ReachConfig, boat_type, build_reach


def gaussian_bumps(sigma: float, corr: float, seed: int):
    """Callable (x, y) -> (ny, nx) bed perturbation: white noise smoothed by a Gaussian of
    standard deviation `corr` (m), rescaled to standard deviation `sigma` (m)."""
    def bumps(x, y):
        dx = float(x[1] - x[0])
        noise = np.random.default_rng(seed).standard_normal((len(y), len(x)))
        field = gaussian_filter(noise, corr / dx, mode="reflect")
        return field * (sigma / field.std())
    return bumps


def config1_case(wall_model: bool = True):
    sec = Section(B=12, Hb=3, z=0, Bf=0, n=0.03)
    boat = BoatType("custom", "long-tail style", hull_L=10.0, hull_B=2.0, draft=0.8, n_props=1, prop_D=0.30,
                    prop_depth=0.35, tilt_deg=12, prop_x=2.5, prop_spacing=0, power_kW=75)
    fleet = Fleet(boat, rows=1, per_row=1, x_first=11.0)
    cfg = ReachConfig(length=48, dx=0.25, cs=0.12, wall_model=wall_model)
    return build_reach(sec, 3.0, 0.8 * 36, 3e-4, fleet, cfg)


def config2_case(seed: int = 2, length: float = 150.0, dx: float = 0.1, with_boat: bool = True):
    h, slope = 4.0, 3e-4
    sec = Section(B=44.0, Hb=4.0, z=2.0, Bf=0.0, n=0.025)
    Q = manning_discharge(sec, h, slope)
    tug = replace(boat_type("tug"), key="tug20", name="pusher tug", hull_L=20.0, hull_B=6.0, draft=1.5,
                  prop_spacing=3.0)
    fleet = Fleet(tug, rows=1, per_row=1, x_first=40.0, enabled=with_boat)
    cfg = ReachConfig(length=length, dx=dx, cs=0.17)
    return build_reach(sec, h, Q, slope, fleet, cfg, bed_bumps=gaussian_bumps(0.15, 5.0, seed))


def config3_inputs(seed: int = 3, dx: float = 0.05):
    """build_reach's arguments for config3_case, as (sec, h, Q, slope, fleet, cfg, bed_bumps)."""
    h, slope = 3.6, 3e-4
    sec = Section(B=60.0 - 2 * 2.0 * h, Hb=h, z=2.0, Bf=0.0, n=0.025)
    Q = manning_discharge(sec, h, slope)
    tug = replace(boat_type("tug"), key="tug20", name="pusher tug", hull_L=20.0, hull_B=6.0, draft=1.5,
                  prop_spacing=3.0)
    fleet = Fleet(tug, rows=1, per_row=1, x_first=40.0)
    cfg = ReachConfig(length=150.0, dx=dx, cs=0.17)
    return sec, h, Q, slope, fleet, cfg, gaussian_bumps(0.15, 5.0, seed)


def config3_case(seed: int = 3, dx: float = 0.05):
    """The 16-bit-storage scale case: the config-2 reach (150 m, 60 m top width, 1:2 banks,
    seeded Gaussian bed bumps, 20 m pusher tug) at a 3.6 m stage and dx = 0.05 m, which the
    reference's grid rule turns into 3000 x 1202 x 72 = 259.6M cells."""
    sec, h, Q, slope, fleet, cfg, bumps = config3_inputs(seed, dx)
    return build_reach(sec, h, Q, slope, fleet, cfg, bed_bumps=bumps)


ENSEMBLE_TYPES = ("longtail", "outboard", "tug", "pontoon", "jet_hp", "jet_mp", "curtain")


def ensemble_case(seed: int, dx: float = 0.1, cells_range=(2.0e6, 2.0e7)):
    """A seeded boat case of the batched-ensemble workload: boat type from ENSEMBLE_TYPES,
    stage 2-5 m, 1-4 boats abreast or in line, propeller tilt 0-20 deg, trapezoidal channel
    (bank slope 0-2, Manning n 0.025-0.035) sized for a lattice of 2M-20M cells at dx."""
    from dataclasses import replace as _replace
    from .reach3d import BOAT_TYPES
    rng = np.random.default_rng(seed)
    h = float(rng.choice([2.0, 3.0, 4.0, 5.0]))
    z = float(rng.choice([0.0, 1.0, 2.0]))
    n = float(rng.uniform(0.025, 0.035))
    target = float(np.exp(rng.uniform(np.log(cells_range[0]), np.log(cells_range[1]))))
    top = float(rng.uniform(20.0, 50.0))
    B = max(top - 2 * z * h, 8.0)
    length = float(np.clip(target * dx ** 3 / ((B + 2 * z * h) * h), 40.0, 400.0))
    key = ENSEMBLE_TYPES[int(rng.integers(len(ENSEMBLE_TYPES)))]
    boat = next(b for b in BOAT_TYPES if b.key == key)
    fit = min(1.0, 0.6 * h / max(boat.draft + boat.prop_depth, 0.5))
    boat = _replace(boat, tilt_deg=float(rng.uniform(0.0, 20.0)) if boat.prop_D > 0 else 0.0,
                    draft=boat.draft * fit, prop_depth=max(boat.prop_depth * fit, 0.4),
                    prop_D=min(boat.prop_D, 0.4 * h), hull_B=min(boat.hull_B, 0.2 * B))
    count = int(rng.integers(1, 5))
    abreast = bool(rng.integers(2))
    if abreast:
        count = min(count, max(1, int(B // (boat.hull_B + 2.0))))
    fleet = Fleet(boat, rows=1 if abreast else count, per_row=count if abreast else 1,
                  row_spacing=boat.hull_L + 10.0, x_first=0.3 * length)
    sec = Section(B=B, Hb=h, z=z, Bf=0.0, n=n)
    Q = manning_discharge(sec, h, 3e-4)
    return build_reach(sec, h, Q, 3e-4, fleet, ReachConfig(length=length, dx=dx, cs=0.17))
