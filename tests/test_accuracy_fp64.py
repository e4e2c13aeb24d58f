"""Water level and bed shear of the B200 path against the FP64 oracle (needs a B200).

The config-1 boat case (192 x 50 x 12, long-tail boat, Manning wall model) is run with
Run3D's cadence -- 20-step chunks, the smoothstep force ramp, the column-mean wall-model
speed refreshed between chunks -- three times: by the CPU oracle in float64, and on the GPU
with float32 and with 16-bit population storage.  Compared quantities, as the reference's
readouts define them (floodsim/reach3d.py:545-568, 571-618):

* the lid water level eta(x), referenced to the outlet: the largest difference along the
  reach, and the upstream level drop eta(x_up) - eta(outlet) that `compare` reports, in cm;
* the bed shear tau = rho cf |u|^2 of the first fluid cell above the bed: its maximum, and
  the mean absolute difference over the bed relative to the mean shear.

The 2000-step run ends inside the force ramp, so the fields are instantaneous.  Each
number is printed; the bounds are the acceptance bars of the 16-bit store (level within
0.5 cm, shear within 2%), and float32 is held to the same bars.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEPS = 2000
LEVEL_CM = 0.5
SHEAR_REL = 0.02


def _oracle_run(reach, steps, precision="f64", average=False):
    """Run3D.advance's chunk loop (water_flow_simulation_b200/reach3d.py) on the oracle; with
    `average`, the float64 sums of rho, ux, |u| and ux^2 over the chunk ends in the averaging
    window (t >= t_avg), as Run3D accumulates them, returned with their count."""
    from oracle.oracle import OracleLBM
    from water_flow_simulation_b200.reach3d import Run3D
    nu_lb = max(1e-6 * reach.dt / reach.dx ** 2, 2e-4)
    uin = (reach.uin_phys / reach.vel).astype(np.float32)
    O = OracleLBM(reach.solid, reach.Fx, reach.Fy, reach.Fz, uin, 0.5 + 3 * nu_lb, reach.cfg.cs, reach.cf,
                  precision=precision)
    F0 = [np.asarray(a, np.float32).ravel() for a in (reach.Fx, reach.Fy, reach.Fz)]
    t_total = reach.cfg.run_flows * reach.cfg.length / max(reach.V, 0.05)
    t_ramp = min(0.15 * t_total, 20.0) if reach.props else 0.0
    t_avg = t_total * (1 - reach.cfg.avg_frac)
    t, k, ramp_done = 0.0, 0, t_ramp <= 0
    scale = np.float32(0.0 if not ramp_done else 1.0)
    sums, navg = None, 0
    while k < steps:
        m = min(Run3D.avg_every, steps - k)
        if not ramp_done:
            f = min(t / t_ramp, 1.0)
            scale = np.float32(f * f * (3 - 2 * f))
            ramp_done = scale >= 1.0
        O.Fx, O.Fy, O.Fz = ((F * scale).astype(O.dt) for F in F0)
        if reach.bedwall is not None:
            O.update_uref(reach.bedwall)
        O.step(m)
        k += m
        t_next = t + m * reach.dt
        if average and t_next >= t_avg:
            u, v, w, r = (np.asarray(a, np.float64) for a in (O.ux, O.uy, O.uz, O.rho))
            add = (r, u, v, w, np.sqrt(u * u + v * v + w * w), u * u)
            sums = list(add) if sums is None else [a + b for a, b in zip(sums, add)]
            navg += 1
        t = t_next
    if average:
        return O, sums, navg
    return O


def _readouts_host(reach, rho, ux, uy, uz, sp=None):
    from water_flow_simulation_b200.accuracy import level_and_shear
    return level_and_shear(reach, rho, ux, uy, uz, sp=sp)


def _errors(reach, eta, tau, eta_ref, tau_ref):
    from water_flow_simulation_b200.accuracy import errors
    return errors(eta, tau, eta_ref, tau_ref)


@pytest.fixture(scope="module")
def config1_runs():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.reach3d import Run3D, profiles_device
    reach = config1_case()
    O64 = _oracle_run(reach, STEPS, "f64")
    ref = _readouts_host(reach, O64.rho, O64.ux, O64.uy, O64.uz)
    out = {}
    for storage in ("fp32", "fp16"):
        run = Run3D(reach, storage=storage)
        run.advance(STEPS)
        p = profiles_device(run, mean=False)
        out[storage] = _errors(reach, p["eta"], p["tau_bed"], *ref)
        # the device readouts against the same readouts of the GPU fields on the host
        L = run.lbm
        host = _readouts_host(reach, *(getattr(L, k).cpu().numpy() for k in ("rho", "ux", "uy", "uz")))
        out[storage + "_readout_check"] = (p["eta"], p["tau_bed"], *host)
    return reach, out


@pytest.mark.parametrize("storage", ("fp32", "fp16"))
def test_level_and_shear_against_fp64_oracle(config1_runs, storage):
    reach, out = config1_runs
    e = out[storage]
    print(f"config-1, {STEPS} steps, {storage} vs FP64 oracle: level max {e['level_max_cm']:.3f} cm, "
          f"upstream drop {e['drop_cm']:.3f} cm, bed shear max {100 * e['shear_max_rel']:.2f} %, "
          f"mean {100 * e['shear_mean_rel']:.2f} %")
    assert e["level_max_cm"] <= LEVEL_CM and e["drop_cm"] <= LEVEL_CM, e
    assert e["shear_max_rel"] <= SHEAR_REL and e["shear_mean_rel"] <= SHEAR_REL, e


@pytest.mark.parametrize("storage", ("fp32", "fp16"))
def test_device_readouts_equal_host_readouts(config1_runs, storage):
    _, out = config1_runs
    eta_d, tau_d, eta_h, tau_h = out[storage + "_readout_check"]
    assert np.abs(eta_d - eta_h).max() <= 1e-9
    assert np.abs(tau_d - tau_h).max() <= 1e-9 * max(tau_h.max(), 1e-30)


@pytest.fixture(scope="module")
def full_case_oracle():
    """The whole config-1 case on the FP64 oracle, with its time averages."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.reach3d import Run3D
    reach = config1_case()
    t_total = reach.cfg.run_flows * reach.cfg.length / max(reach.V, 0.05)
    steps = int(np.ceil(t_total / reach.dt / Run3D.avg_every)) * Run3D.avg_every
    _, sums, navg = _oracle_run(reach, steps, "f64", average=True)
    r, u, v, w, sp, _ = (a / navg for a in sums)
    return reach, steps, navg, _readouts_host(reach, r, u, v, w, sp=sp)


@pytest.mark.parametrize("storage", ("fp32", "fp16"))
def test_full_case_time_averages_against_fp64_oracle(full_case_oracle, storage):
    """The whole config-1 case (t_total = one flow-through, ~18.4k steps) and the reference's
    time-averaged readouts over its trailing window: lid level eta(x) and bed shear from the
    mean speed, against the same averages of an FP64 oracle run."""
    from water_flow_simulation_b200.reach3d import Run3D, profiles_device
    reach, steps, navg, ref = full_case_oracle
    run = Run3D(reach, storage=storage)
    run.advance(steps)
    p = profiles_device(run, mean=True)
    assert navg == run.navg > 0
    e = _errors(reach, p["eta"], p["tau_bed"], *ref)
    print(f"config-1 full case ({steps} steps, {navg} averaged outputs), {storage} vs FP64 oracle: level max "
          f"{e['level_max_cm']:.3f} cm, upstream drop {e['drop_cm']:.3f} cm, bed shear max "
          f"{100 * e['shear_max_rel']:.2f} %, mean {100 * e['shear_mean_rel']:.2f} %")
    assert e["level_max_cm"] <= LEVEL_CM and e["drop_cm"] <= LEVEL_CM, e
    assert e["shear_max_rel"] <= SHEAR_REL and e["shear_mean_rel"] <= SHEAR_REL, e
