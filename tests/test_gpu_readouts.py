"""FP64 device readouts (lbm_profiles) against the host restatement of floodsim/reach3d.py:545-568.

profiles() reduces the fields with NumPy on the host in float32, exactly as the reference
does; profiles_device() reduces them on the device in float64.  They agree to float32
summation accuracy (1e-5 relative to each profile's scale); the bed-shear maps are
elementwise maxima of the same values and agree to float32 rounding.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(steps=3, chunk=20):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.reach3d import Run3D
    run = Run3D(config1_case())
    run.lbm.force_scale = 1.0
    for _ in range(steps):
        run.lbm.step(chunk, accumulate=True)
        run.navg += 1
    torch.cuda.synchronize()
    return run


def _close(a, b, rel=1e-5):
    scale = max(float(np.abs(b).max()), 1e-30)
    return float(np.abs(np.asarray(a) - np.asarray(b)).max()) <= rel * scale


def test_profiles_device_matches_host_profiles():
    from water_flow_simulation_b200.reach3d import profiles, profiles_device
    run = _run()
    host = profiles(run)
    dev = profiles_device(run)
    for k in ("us", "umax", "q", "mom", "tau_max_x"):
        assert _close(dev[k], host[k]), k
    # eta is a difference of two lid levels: compare against the level scale, not its own range
    level_scale = float(np.abs(run.field("rho", mean=True)).max())
    assert float(np.abs(dev["eta"] - host["eta"]).max()) <= 1e-5 * max(level_scale, 1e-6)
    assert _close(dev["tau_bed"], host["tau_bed"], rel=1e-6)
    assert dev["fluid_cells"] == float((~run.r.solid).sum())


def test_profile_sums_of_instantaneous_fields():
    run = _run(steps=1)
    L = run.lbm
    s = L.profile_sums(mean=False)
    solid = run.r.solid
    fl = ~solid
    ux = L.ux.cpu().numpy().reshape(solid.shape).astype(np.float64)
    rho = L.rho.cpu().numpy().reshape(solid.shape).astype(np.float64)
    np.testing.assert_allclose(s["q"], (ux * fl).sum(axis=(0, 1)), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(s["drho"], ((rho - 1) * fl).sum(axis=(0, 1)), rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(s["top_n"], fl[-1].sum(0))
    np.testing.assert_allclose(s["n_fluid"], fl.sum(axis=(0, 1)))
    assert abs(s["mass"].sum() - (rho * fl).sum()) <= 1e-9 * (rho * fl).sum()


def test_profiles_are_deterministic():
    run = _run(steps=1)
    a = run.lbm.profile_sums(mean=True)
    b = run.lbm.profile_sums(mean=True)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
