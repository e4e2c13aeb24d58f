"""Host logic of the accuracy statements (accuracy.py) on the CPU: the reference's readouts
from fields, the error measures, and the boat's level change from saved profiles."""
import numpy as np

from water_flow_simulation_b200.accuracy import errors, level_and_shear, level_change


def test_errors_of_identical_and_shifted_profiles():
    x = np.linspace(0, 1, 50)
    eta = 0.05 * (1 - x)
    tau = 1.0 + x
    e = errors(eta, tau, eta, tau)
    assert e == dict(level_max_cm=0.0, drop_cm=0.0, shear_max_rel=0.0, shear_avg_rel=0.0, shear_mean_rel=0.0)
    e = errors(eta + 0.002, tau * 1.01, eta, tau)
    assert abs(e["level_max_cm"] - 0.2) < 1e-12 and e["drop_cm"] < 1e-12      # an offset leaves the drop
    assert abs(e["shear_max_rel"] - 0.01) < 1e-12 and abs(e["shear_mean_rel"] - 0.01) < 1e-12
    assert abs(e["shear_avg_rel"] - 0.01) < 1e-12


def test_level_and_shear_of_a_uniform_state():
    """Rest density 1 and a uniform stream: level 0 everywhere, shear only on first fluid cells."""
    from water_flow_simulation_b200.cases import config1_case
    r = config1_case()
    n = r.solid.size
    fl = ~r.solid.ravel()
    eta, tau = level_and_shear(r, np.ones(n), 0.05 * fl, np.zeros(n), np.zeros(n))
    assert eta.shape == (r.nx,) and np.all(eta == 0)
    assert tau.shape == (r.ny, r.nx) and tau.max() > 0 and np.all(tau >= 0)


def test_level_change_from_saved_profiles(tmp_path):
    from water_flow_simulation_b200.cases import config1_case
    r = config1_case()
    x = r.x
    base = 0.03 * (1 - x / x[-1])
    boat = base + 0.01 * (x < 20)
    np.savez(tmp_path / "boat.npz", x=x, fp64_eta=boat, fp16_eta=boat + 0.001 * (x < 20), fp64_tau=x, fp16_tau=x)
    np.savez(tmp_path / "base.npz", x=x, fp64_eta=base, fp16_eta=base, fp64_tau=x, fp16_tau=x)
    d = level_change(tmp_path / "boat.npz", tmp_path / "base.npz", r)
    assert abs(d["fp64"]["d_eta_cm"] - 1.0) < 1e-9 and d["fp64"]["error_cm"] == 0.0
    assert abs(d["fp16"]["error_cm"] - 0.1) < 1e-9        # a uniform offset would cancel; a drop does not


def test_boat_effects_equal_compare_of_the_saved_profiles(tmp_path):
    """The statement's boat effects (level change, discharge gain from the momentum balance, net
    force, surface-speed gain, largest shear and speed) are compare() of the saved boat and base
    profiles; float64's own errors are 0 and another run's are its differences from float64."""
    import json
    import os
    from golden_io import GOLDEN
    from test_reach_builder import build_from_spec
    from water_flow_simulation_b200.accuracy import EFFECT_KEYS, PROFILE_SAVE, boat_effects
    from water_flow_simulation_b200.reach3d import AVG_KEYS, compare, profiles_from_sums
    d = np.load(os.path.join(GOLDEN, "readouts_mini_tug.npz"))
    r = build_from_spec(json.loads(str(d["spec"])))
    rb = build_from_spec(json.loads(str(d["base_spec"])))
    prof = {tag: profiles_from_sums(reach, {k: d[f"{tag}_sum_{k}"] for k in AVG_KEYS}, int(d[f"{tag}_navg"]))
            for tag, reach in (("boat", r), ("base", rb))}
    scaled = {tag: dict(p, mom=p["mom"] * 1.01) for tag, p in prof.items()}    # a second "run"
    for tag in ("boat", "base"):
        saved = {}
        for run, p in (("fp64", prof[tag]), ("fp16", scaled[tag])):
            saved.update({f"{run}_prof_{n}": np.asarray(p[n]) for n in PROFILE_SAVE})
        np.savez(tmp_path / f"{tag}.npz", **saved)
    eff = boat_effects(tmp_path / "boat.npz", tmp_path / "base.npz", r)
    want = compare(prof["boat"], prof["base"], r, r.cfg)
    for n in EFFECT_KEYS:
        assert eff["fp64"][n] == float(want[n]) and eff["fp64"]["error"][n] == 0.0, n
    got = compare(scaled["boat"], scaled["base"], r, r.cfg)
    assert eff["fp16"]["dQ_net_pct"] == float(got["dQ_net_pct"])
    assert abs(eff["fp16"]["error"]["dQ_net_pct"] - (got["dQ_net_pct"] - want["dQ_net_pct"])) < 1e-12
