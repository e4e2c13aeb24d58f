"""The web viewer's case export (floodsim/web3d.py:35-86) on the CPU: the oracle's int8
velocity blocks against the reference's own exports (tests/golden/export_*.npz), and the
host part of export.export_case -- bed heights, pooled shear, profiles, hulls, props --
against the same exports, with the velocity blocks taken from the oracle."""
import json

import numpy as np
import pytest

from golden_io import GOLDEN, Case
from test_reach_builder import build_from_spec

EXPORT_CASES = ("mini_cfg1", "mini_tug", "jet_flood")


def _case(name):
    c = Case(f"{GOLDEN}/export_{name}.npz")
    d = c.d
    sums = [d["sum_ux"], d["sum_uy"], d["sum_uz"]]
    res = dict(x=d["res_x"], eta=d["res_eta"], umax=d["res_umax"], tau_bed=d["res_tau_bed"])
    return c, sums, int(d["navg"]), res, json.loads(str(d["export"]))


@pytest.mark.parametrize("name", EXPORT_CASES)
def test_oracle_velocity_blocks_equal_reference_export(name):
    import base64
    from oracle.export_oracle import velocity_int8
    c, sums, navg, _, ref = _case(name)
    q, scale, sp99 = velocity_int8(sums, navg, c.dx / c.dt, c.solid)
    assert q.shape == (c.nz, c.ny // 2, c.nx // 2, 3)
    assert base64.b64encode(q.tobytes()).decode() == ref["u"]
    assert scale == ref["scale"] and sp99 == ref["sp99"]
    assert (q == -128).any() and (np.abs(q[q != -128]) <= 126).all()


@pytest.mark.parametrize("name", EXPORT_CASES)
def test_host_part_of_export_equals_reference(name, monkeypatch):
    from oracle.export_oracle import velocity_int8
    from water_flow_simulation_b200 import export
    c, sums, navg, res, ref = _case(name)
    reach = build_from_spec(c.spec)
    assert np.array_equal(reach.solid, c.solid)
    monkeypatch.setattr(export, "velocity_int8",
                        lambda run: velocity_int8(sums, navg, run.r.vel, run.r.solid))
    run = type("Run", (), {"r": reach, "navg": navg})()
    out = json.loads(json.dumps(export.export_case(run, "case", None, res)))
    # the boat catalogue's display names are English here (the reference's are Thai)
    assert out.pop("boat") == (reach.fleet.boat.name if reach.fleet.enabled else "")
    ref.pop("boat")
    assert out == ref
