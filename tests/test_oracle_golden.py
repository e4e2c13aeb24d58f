"""The CPU oracle against the reference's own Numba solver outputs (golden fixtures).

The fixtures were produced by the reference (floodsim/lbm3d.py Numba path driven by
floodsim/reach3d.py Run3D.advance); the oracle must reproduce them bit for bit.
"""
import numpy as np
import pytest

from golden_io import ADVANCE_CASES, STEP_CASES, STEP_NS, load_advance_case, load_step_case
from oracle.oracle import OracleLBM, OracleRun3D, equilibrium_init


def _oracle(c, precision="f32"):
    o = OracleLBM(c.solid, *c.F, c.uin_lb, c.tau0, c.cs, c.cf, precision=precision)
    o.csmag2 = float(c.d["csmag2"])
    return o


@pytest.mark.parametrize("name", STEP_CASES)
def test_oracle_matches_reference_bit_exact(name):
    c = load_step_case(name)
    o = _oracle(c)
    done = 0
    for n in STEP_NS:
        # Run3D.advance refreshes uref before each call's first chunk (reach3d.py:438-440)
        if c.bedwall is not None:
            o.update_uref(c.bedwall)
        o.step(n - done)
        done = n
        ref = c.state(n)
        for k in ("rho", "ux", "uy", "uz"):
            assert np.array_equal(getattr(o, k), ref[k]), (name, n, k)
        if n == 1:
            fl = np.tile(~c.solid.ravel(), 19)      # solid cells of fd are never written by the reference
            assert np.array_equal(o.f[fl], c.d["f_1"][fl])
    if c.bedwall is not None:
        # the last refresh in both runs came from the step-5 fields, before the 20-step chunk
        assert np.array_equal(o.uref, c.d["uref_25"])


def test_equilibrium_init_is_reference_start():
    c = load_step_case("mini_cfg1")
    f0 = equilibrium_init(c.solid, c.uin_lb)
    # one step from f0 reproduces the stored state, so f0 is the reference start; also check its moments
    n = c.N
    rho = f0.reshape(19, n).sum(0)
    assert np.allclose(rho, 1.0, atol=2e-7)


@pytest.mark.parametrize("name", ("mini_cfg1", "mini_tug"))
def test_fp64_oracle_tracks_fp32(name):
    c = load_step_case(name)
    o32, o64 = _oracle(c), _oracle(c, "f64")
    for _ in range(5):
        if c.bedwall is not None:
            o32.update_uref(c.bedwall)
            o64.update_uref(c.bedwall)
        o32.step(1)
        o64.step(1)
    umax = np.abs(o64.ux).max()
    assert np.abs(o32.ux - o64.ux).max() / umax < 1e-4
    assert np.abs(o32.rho - o64.rho).max() < 1e-5


def oracle_run3d(c):
    """OracleRun3D of an advance fixture, with the fixture's moved ramp time and averaging start."""
    return OracleRun3D(c.solid, *c.F, c.uin_lb, c.tau0, c.cs, c.cf, c.bedwall, c.dt, float(c.d["t_ramp"]),
                       float(c.d["t_avg"]))


@pytest.mark.parametrize("name", ADVANCE_CASES)
def test_oracle_run3d_advance_matches_reference_bit_exact(name):
    """Force ramp, uref cadence and float32 time-average sums of Run3D.advance
    (floodsim/reach3d.py:424-453): every chunk's fields, uref and sums equal the reference's."""
    c = load_advance_case(name)
    o = oracle_run3d(c)
    for k, m in enumerate(c.d["chunks"]):
        o.advance(int(m))
        for nm in ("rho", "ux", "uy", "uz", "uref"):
            assert np.array_equal(getattr(o.lbm, nm), c.d[f"{nm}_c{k}"]), (name, k, nm)
        assert o.navg == int(c.d[f"navg_c{k}"])
        for nm in OracleRun3D.AVG_KEYS:
            assert np.array_equal(o.sum[nm], c.d[f"sum_{nm}_c{k}"]), (name, k, nm)
    # the ramp was inside (0, 1) in some chunk and complete by the last one
    scales = [float(c.d[f"fx_scale_c{k}"]) for k in range(len(c.d["chunks"]))]
    assert scales[0] == 0.0 and any(0 < s < 1 for s in scales) and scales[-1] == 1.0
