"""The host reach builder against the reference's build_reach/wall_cf outputs (golden fixtures).

Every array and scalar must be identical: the lattice dims, dt, the solid mask, the
1/7-power inlet profile, the actuator-disk/jet forces, the wall friction and the
bed/bank mask (floodsim/reach3d.py:201-343).
"""
import json
from dataclasses import replace

import numpy as np
import pytest

from golden_io import REACH_CASES, STEP_CASES, load_reach_case, load_step_case
from water_flow_simulation_b200.geometry import Section
from water_flow_simulation_b200.reach3d import BoatType, Fleet, ReachConfig, boat_type, build_reach


def build_from_spec(spec):
    key, over = spec["boat"]
    b = BoatType("custom", **over) if key == "custom" else replace(boat_type(key), **over)
    return build_reach(Section(**spec["sec"]), spec["h"], spec["Q"], spec["S"], Fleet(b, **spec["fleet"]),
                       ReachConfig(**spec["cfg"]))


def _check(c):
    r = build_from_spec(c.spec)
    assert (r.nx, r.ny, r.nz) == (c.nx, c.ny, c.nz)
    nu_lb = max(1e-6 * r.dt / r.dx ** 2, 2e-4)
    got = [r.dx, r.dt, r.V, r.A, r.W, r.h, r.Q, r.S, 0.5 + 3 * nu_lb, r.cfg.cs]
    assert np.array_equal(np.array(got), np.array([c.dx, c.dt, c.V, c.A, c.W, c.h, c.Q, c.S, c.tau0, c.cs]))
    assert np.array_equal(r.solid, c.solid)
    assert np.array_equal(r.uin_phys, c.uin_phys)
    assert np.array_equal((r.uin_phys / r.vel).astype(np.float32), c.uin_lb)
    for a, b in zip((r.Fx, r.Fy, r.Fz), c.F):
        assert a.dtype == np.float32 and np.array_equal(a, b)
    if c.cf is None:
        assert r.cf is None and r.bedwall is None
    else:
        assert r.cf.dtype == np.float32 and np.array_equal(r.cf, c.cf)
        assert np.array_equal(r.bedwall, c.bedwall)
    assert [list(map(float, h)) for h in r.hulls] == c.meta["hulls"]
    props = {str(i): {k: float(v) for k, v in p.items()} for i, p in enumerate(r.props)}
    assert props == c.meta["props"]
    assert len(r.notes) == len(c.meta["notes"])


@pytest.mark.parametrize("name", REACH_CASES)
def test_reach_bit_exact(name):
    _check(load_reach_case(name))


@pytest.mark.parametrize("name", STEP_CASES)
def test_step_case_inputs_bit_exact(name):
    _check(load_step_case(name))


def test_boat_physics_catalogue():
    """Thrust and jet speed of the catalogue boats (floodsim/reach3d.py:48-72)."""
    tug = boat_type("tug")
    assert abs(tug.thrust() - (2 * 1000.0 * np.pi * 1.2 ** 2 / 4 * (0.6 * 300e3) ** 2) ** (1 / 3)) < 1e-9
    jet = boat_type("jet_hp")
    assert abs(jet.jet_speed() - np.sqrt(2 * 100e5 / 1000.0)) < 1e-12
    assert abs(jet.thrust() - 2 * 0.7 * 25e3 / jet.jet_speed()) < 1e-12
    assert abs(jet.thrust() - 1000.0 * np.pi * jet.outlet_D() ** 2 / 4 * jet.jet_speed() ** 2) < 1e-9
    with pytest.raises(KeyError):
        boat_type("submarine")
