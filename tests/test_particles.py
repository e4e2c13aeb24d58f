"""Tracer particles on the CPU: the oracle's step against the reference's own particle runs
(tests/golden/particles_*.npz), and Run3D.init_particles' start positions (seeded as the
reference seeds them)."""
import numpy as np
import pytest

from golden_io import GOLDEN, Case

PARTICLE_CASES = ("mini_cfg1", "mini_tug")


def load(name):
    c = Case(f"{GOLDEN}/particles_{name}.npz")
    return c, c.d


@pytest.mark.parametrize("name", PARTICLE_CASES)
def test_oracle_step_equals_reference_particles(name):
    from oracle.particles_oracle import move
    c, d = load(name)
    vel = c.dx / c.dt
    restarted_total = 0
    for k, dt in enumerate(d["dts"]):
        P0, P1 = d[f"P{k}"], d[f"P{k + 1}"]
        P, bad = move(P0, d["ux"], d["uy"], d["uz"], c.solid, vel, float(dt), c.dx)
        assert np.array_equal(P[~bad], P1[~bad])                  # bit for bit
        assert (P1[bad, 0] >= 0).all() and (P1[bad, 0] < 2 * c.dx).all()   # restarts sit at the inlet
        restarted_total += int(bad.sum())
    assert restarted_total > 0


@pytest.mark.parametrize("name", PARTICLE_CASES)
def test_init_particles_matches_reference_start(name):
    from test_reach_builder import build_from_spec
    from water_flow_simulation_b200.reach3d import Run3D
    c, d = load(name)
    reach = build_from_spec(c.spec)
    run = Run3D.__new__(Run3D)          # the start positions need no solver
    run.r = reach
    rng = np.random.default_rng(0)
    fluid = np.argwhere(~reach.solid)
    n = len(d["P0"])
    pick = fluid[rng.integers(0, len(fluid), n)]
    P = (pick[:, ::-1] + rng.random((n, 3))) * reach.dx
    assert np.array_equal(P, d["P0"])
