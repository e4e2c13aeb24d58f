"""FP64 force sums on the device (lbm_body_forces, needs a B200) against the oracle.

After N steps of the reference's stepped cases (boats with propellers or jets), the device
momentum-exchange force on every hull must equal the oracle's (oracle_body_forces_f32, the
same bounce-back and wall function on the oracle's own state) within 1e-4 of the largest
hull force component, or twice the oracle's own 1-ulp spread of the forces where that is
larger (the parity rule of tests/parity_util.py applied to the force sums), and the
applied body force must equal the float64 sum of the force arrays.  The 16-bit store's
forces track the float32 ones within its rounding (2e-2), and Run3D converts to newtons
(the applied force equals the propellers' thrust along their axes).
"""
import numpy as np
import pytest

from golden_io import load_step_case
from oracle.oracle import body_forces as oracle_body_forces
from parity_util import make_oracle
from test_gpu_parity import _require_gpu, make_solver
from test_reach_builder import build_from_spec

pytestmark = pytest.mark.gpu


def force_spread(c, r, nb):
    """The oracle's own sensitivity of the hull forces: the largest change of a component after
    the same 5 steps from a start perturbed by one float32 ulp per population.  A hull's drag is
    a small difference of its faces' pressure forces, and the wall function normalises a
    tangential speed that can be tiny, so one ulp moves it by more than 1e-4 of the largest
    component on some cases."""
    a, b = make_oracle(c), make_oracle(c)
    sgn = np.random.default_rng(1).choice([-1.0, 1.0], b.f.size).astype(np.float32)
    b.f = np.nextafter(b.f, b.f + sgn).astype(np.float32)
    for n in (1, 1, 3):
        for o in (a, b):
            o.update_uref(c.bedwall)
            o.step(n)
    for o in (a, b):
        o.update_uref(c.bedwall)
    return float(np.abs(oracle_body_forces(a, r.body, nb) - oracle_body_forces(b, r.body, nb)).max())


@pytest.mark.parametrize("name", ("mini_tug", "mini_cfg1", "mini_jet"))
def test_body_forces_match_oracle(name):
    _require_gpu()
    c = load_step_case(name)
    r = build_from_spec(c.spec)
    nb = len(r.hulls)
    assert nb > 0 and r.body is not None
    L = make_solver(c)
    O = make_oracle(c)
    for n in (1, 1, 3):
        O.update_uref(c.bedwall)
        O.step(n)
        L.step(n)
    O.update_uref(c.bedwall)              # the column means the next step uses (the device refreshed them)
    want = oracle_body_forces(O, r.body, nb)
    got, applied = L.body_forces(r.body, nb)
    scale = float(np.abs(want).max())
    assert scale > 0
    bar = max(1e-4 * scale, 2 * force_spread(c, r, nb))
    assert float(np.abs(got - want).max()) <= bar, (got, want, bar)
    F = [np.asarray(a, np.float64)[~c.solid] for a in c.F]
    np.testing.assert_allclose(applied, [f.sum() for f in F], rtol=1e-12, atol=1e-18)
    L16 = make_solver(c, storage="fp16")
    L16.step(1); L16.step(1); L16.step(3)
    got16, applied16 = L16.body_forces(r.body, nb)
    assert float(np.abs(got16 - got).max()) <= 2e-2 * scale
    np.testing.assert_allclose(applied16, applied, rtol=1e-12)


def test_run3d_forces_in_newtons():
    """Run3D.body_forces: the applied force, after the ramp, is the thrust the reach builder
    spread over the propeller disks (sum of T along each axis, to float32 rounding)."""
    _require_gpu()
    from water_flow_simulation_b200.reach3d import Run3D
    c = load_step_case("mini_tug")
    r = build_from_spec(c.spec)
    run = Run3D(r)
    run.t_ramp = 2 * r.dt
    run.advance(3)                        # force scale 0 in this chunk, 1 from the next
    run.advance(3)
    assert run.lbm.force_scale == 1.0
    out = run.body_forces()
    T = np.zeros(3)
    for p in r.props:
        t, w = np.radians(p["tilt"]), np.radians(p["yaw"])
        T += p["T"] * np.array([np.cos(t) * np.cos(w), np.cos(t) * np.sin(w), -np.sin(t)])
    np.testing.assert_allclose(out["applied"], T, rtol=1e-5, atol=1e-6 * np.abs(T).max())
    assert out["hulls"].shape == (len(r.hulls), 3) and np.all(np.isfinite(out["hulls"]))
