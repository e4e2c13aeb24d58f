"""Tracer particles on the device (lbm_move_particles, Run3D.move_particles) against the CPU
oracle and the reference's particle runs (needs a B200)."""
import numpy as np
import pytest

from test_particles import PARTICLE_CASES, load
from test_reach_builder import build_from_spec

pytestmark = pytest.mark.gpu


def _run_with_fields(name, seed=7):
    import torch
    from water_flow_simulation_b200.reach3d import Run3D
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    c, d = load(name)
    reach = build_from_spec(c.spec)
    run = Run3D(reach)
    L = run.lbm
    for nm in ("ux", "uy", "uz"):
        dst = getattr(L, "_" + nm).view(L.nz, L.ny, L.pitch)[..., :L.nx]
        dst.copy_(torch.from_numpy(d[nm].reshape(L.nz, L.ny, L.nx)))
    run.init_particles(len(d["P0"]), seed=seed)
    return c, d, reach, run


@pytest.mark.parametrize("name", PARTICLE_CASES)
def test_device_particles_against_oracle_and_reference(name):
    from oracle.particles_oracle import move
    c, d, reach, run = _run_with_fields(name)
    assert np.array_equal(run.P.cpu().numpy(), d["P0"])            # the reference's start positions
    inlet_fluid = ~reach.solid[:, :, 1]
    total = 0
    for k, dt in enumerate(d["dts"]):
        P0 = run.P.cpu().numpy()
        run.move_particles(float(dt))
        P1 = run.P.cpu().numpy()
        P, bad = move(P0, d["ux"], d["uy"], d["uz"], reach.solid, reach.vel, float(dt), reach.dx)
        assert np.array_equal(P1[~bad], P[~bad])
        if k == 0:                                                 # same start: same moves as the reference
            assert np.array_equal(P1[~bad], d["P1"][~bad])
        R = P1[bad]
        assert (R[:, 0] >= 0).all() and (R[:, 0] < 2 * reach.dx).all()
        iy, iz = (R[:, 1] / reach.dx).astype(int), (R[:, 2] / reach.dx).astype(int)
        assert inlet_fluid[iz, iy].all()                            # restarted inside a fluid inlet cell
        total += int(bad.sum())
    assert total > 0 and int(run._respawned.item()) == total


def test_device_particles_reproducible_from_seed():
    runs = [_run_with_fields("mini_tug", seed=s) for s in (11, 11, 12)]
    out = []
    for _, d, _, run in runs:
        for dt in d["dts"]:
            run.move_particles(float(dt))
        out.append(run.P.cpu().numpy())
    assert np.array_equal(out[0], out[1])
    assert not np.array_equal(out[0], out[2])
    x, y, z = runs[0][3].particles_xyz()
    r = runs[0][2]
    assert np.array_equal(y, out[0][:, 1] + r.y[0] - 0.5 * r.dx)
