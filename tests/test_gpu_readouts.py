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


@pytest.mark.parametrize("name", ("mini_tug", "mini_cfg1"))
def test_profiles_device_matches_reference_profiles(name):
    """The float64 device reductions of the reference's own seeded time-average sums
    (tests/golden/readouts_*.npz) against the reference's float32 profiles of those sums:
    within float32 summation accuracy (1e-5 of each profile's scale; eta within the float32
    rounding of the mean density plus 1e-5 of the level scale), bed shear to float32 rounding; and compare() of the device profiles reproduces the
    reference's level change and net force within that accuracy."""
    import json
    import os
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from golden_io import GOLDEN
    from test_reach_builder import build_from_spec
    from water_flow_simulation_b200.reach3d import AVG_KEYS, Run3D, compare, profiles_device
    d = np.load(os.path.join(GOLDEN, f"readouts_{name}.npz"))
    runs = {}
    for tag, spec in (("boat", json.loads(str(d["spec"]))), ("base", json.loads(str(d["base_spec"])))):
        r = build_from_spec(spec)
        run = Run3D(r)
        L = run.lbm
        avg = L._avg.view(6, L.nz, L.ny, L.pitch)
        for i, k in enumerate(AVG_KEYS):
            avg[i, ..., :L.nx].copy_(torch.as_tensor(d[f"{tag}_sum_{k}"].reshape(L.nz, L.ny, L.nx), device=L.device))
        run.navg = L.navg = int(d[f"{tag}_navg"])
        res = profiles_device(run)
        for k in ("us", "umax", "q", "mom", "tau_max_x"):
            assert _close(res[k], d[f"{tag}_res_{k}"]), (tag, k)
        # the reference rounds each mean density (~1) to float32 before subtracting 1: one float32
        # ulp of rho at each of the two levels eta(x) - eta(outlet), plus summation accuracy
        to_m = r.vel ** 2 / 3.0 / 9.81
        level_scale = float(np.abs(d[f"{tag}_sum_rho"] / L.navg - 1.0).max()) * to_m
        tol = 2 * 2.0 ** -23 * to_m + 1e-5 * level_scale
        assert float(np.abs(res["eta"] - d[f"{tag}_res_eta"]).max()) <= tol, tag
        assert _close(res["tau_bed"], d[f"{tag}_res_tau_bed"], rel=1e-6), tag
        runs[tag] = (r, res)
    (r, res), (_, base) = runs["boat"], runs["base"]
    c = compare(res, base, r, r.cfg)
    want = json.loads(str(d["compare"]))
    assert abs(c["F_net_kN"] - want["F_net_kN"]) <= 1e-4 * max(abs(want["F_net_kN"]), 1.0)
    # four levels enter d_eta: four float32 ulps of the mean density, in cm
    assert abs(c["d_eta_cm"] - want["d_eta_cm"]) <= 100 * 4 * 2.0 ** -23 * r.vel ** 2 / 3.0 / 9.81 + 1e-3
    assert c["jet_reach"] == want["jet_reach"] and c["reach_capped"] == want["reach_capped"]
