"""Run3D.advance against the reference's own advance (needs a B200).

tests/golden/advance_*.npz hold the reference's Run3D.advance (floodsim/reach3d.py:424-453)
in four 3-step chunks with its force ramp moved to 7 steps and its averaging to start at
step 5, so that the chunks cover zero force, two ramp fractions in (0, 1), full force, and
three averaged outputs.  The oracle reproduces those fixtures bit for bit
(tests/test_oracle_golden.py).  Here Run3D -- the ramp applied as the kernel's force scale,
the column-mean uref refreshed by the last step of every chunk, the sums added by that step
-- must match them after every chunk:

* fields within 1e-5 of max|u| and 1e-5 absolute in density, or twice the oracle's own
  1-ulp spread of the same run where that is larger;
* the wall-model speed uref that the next chunk uses, within the same bar;
* navg equal, and each of the six float32 sums within 1e-5 of its largest magnitude
  (velocity sums) or of the density sum's deviation scale;
* the 16-bit store: within its accumulated rounding (3e-2 of max|u| after 12 steps).
"""
import numpy as np
import pytest

from golden_io import ADVANCE_CASES, load_advance_case
from oracle.oracle import OracleRun3D
from parity_util import rel_u_error
from test_gpu_parity import _require_gpu
from test_reach_builder import build_from_spec

pytestmark = pytest.mark.gpu

TOL_U = 1e-5
TOL_RHO = 1e-5
_SPREAD = {}


def _oracle(c):
    return OracleRun3D(c.solid, *c.F, c.uin_lb, c.tau0, c.cs, c.cf, c.bedwall, c.dt, float(c.d["t_ramp"]),
                       float(c.d["t_avg"]))


def spread(name, c):
    """Per-chunk 1-ulp sensitivity of the oracle's Run3D on the fixture's run."""
    if name not in _SPREAD:
        a, b = _oracle(c), _oracle(c)
        sgn = np.random.default_rng(1).choice([-1.0, 1.0], b.lbm.f.size).astype(np.float32)
        b.lbm.f = np.nextafter(b.lbm.f, b.lbm.f + sgn).astype(np.float32)
        out = []
        for m in c.d["chunks"]:
            a.advance(int(m))
            b.advance(int(m))
            out.append(rel_u_error(b.lbm, a.lbm))
        _SPREAD[name] = out
    return _SPREAD[name]


def make_run(c, storage):
    from water_flow_simulation_b200.reach3d import Run3D
    r = build_from_spec(c.spec)
    run = Run3D(r, storage=storage)
    assert not run._ramp_done and run.lbm.force_scale == 0.0
    run.t_ramp = float(c.d["t_ramp"])
    run.t_avg = float(c.d["t_avg"])
    return run


def state(c, k):
    return {nm: c.d[f"{nm}_c{k}"] for nm in ("rho", "ux", "uy", "uz")}


@pytest.mark.parametrize("name", ADVANCE_CASES)
def test_advance_ramp_uref_and_averages_match_reference(name):
    _require_gpu()
    from water_flow_simulation_b200.reach3d import AVG_KEYS
    c = load_advance_case(name)
    run = make_run(c, "fp32")
    L = run.lbm
    chunks = [int(m) for m in c.d["chunks"]]
    sp = spread(name, c)
    for k, m in enumerate(chunks):
        run.advance(m)
        got = {nm: getattr(L, nm).cpu().numpy() for nm in ("rho", "ux", "uy", "uz")}
        want = state(c, k)
        bar = max(TOL_U, 2 * sp[k])
        eu = rel_u_error(got, want)
        er = float(np.abs(got["rho"] - want["rho"]).max())
        assert eu < bar and er < TOL_RHO, (name, k, eu, er, bar)
        # the ramp scale the kernel used in this chunk is the reference's float32 fraction
        assert np.float32(L.force_scale) == np.float32(c.d[f"fx_scale_c{k}"]) or \
            abs(L.force_scale - float(c.d[f"fx_scale_c{k}"])) < 1e-6, (k, L.force_scale)
        assert run.navg == int(c.d[f"navg_c{k}"])
        if k + 1 < len(chunks):
            # uref refreshed at the end of this chunk = the reference's uref for the next chunk
            uref = L.uref.cpu().numpy()
            want_u = c.d[f"uref_c{k + 1}"]
            scale = max(float(np.abs(want_u).max()), 1e-30)
            assert float(np.abs(uref - want_u).max()) / scale < bar, (name, k)
        if run.navg:
            for nm in AVG_KEYS:
                s = L.avg_sum(nm).cpu().numpy()
                w = c.d[f"sum_{nm}_c{k}"]
                if nm == "rho":
                    err = float(np.abs(s - w).max()) / run.navg
                    assert err < TOL_RHO, (name, k, nm, err)
                else:
                    err = float(np.abs(s - w).max()) / max(float(np.abs(w).max()), 1e-30)
                    assert err < bar, (name, k, nm, err, bar)
    assert L.status() == 0


@pytest.mark.parametrize("name", ADVANCE_CASES)
def test_advance_fp16_tracks_reference(name):
    """The 16-bit store through the same chunks, with the same navg, stays within its rounding
    of the reference's run: each step rounds every deviation f - w to 11 significant bits
    (~1e-4 of max|u| in the fields), which the wall-function cells amplify; after the 12 steps
    of this run on mini_tug the fields differ from the reference by 1.5e-2 of max|u|
    (measured on a B200), so the bar is 3e-2 of max|u| and 5e-4 in density."""
    _require_gpu()
    c = load_advance_case(name)
    run = make_run(c, "fp16")
    for k, m in enumerate(int(m) for m in c.d["chunks"]):
        run.advance(m)
        got = {nm: getattr(run.lbm, nm).cpu().numpy() for nm in ("rho", "ux", "uy", "uz")}
        assert rel_u_error(got, state(c, k)) < 3e-2
        assert float(np.abs(got["rho"] - state(c, k)["rho"]).max()) < 5e-4
        assert run.navg == int(c.d[f"navg_c{k}"])
    assert run.lbm.status() == 0
