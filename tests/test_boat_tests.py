"""The boat-test catalogue and runner's host logic (floodsim/boat_tests.py) on the CPU."""
import pytest

from water_flow_simulation_b200.boat_tests import BOAT_TESTS, _variant_reaches, pick_level
from water_flow_simulation_b200.geometry import Section, manning_discharge
from water_flow_simulation_b200.reach3d import BOAT_TYPES, ReachConfig


def test_catalogue_matches_reference_structure():
    assert [t["key"] for t in BOAT_TESTS] == ["B1", "B2", "B3", "B4", "B5", "B6"]
    assert [len(t["variants"]) for t in BOAT_TESTS] == [4, 4, 3, 3, 3, 5]
    keys = {b.key for b in BOAT_TYPES}
    for t in BOAT_TESTS:
        for v in t["variants"]:
            assert v["boat"] in keys and v["rows"] >= 1 and v["per_row"] >= 1


def test_pick_level():
    lv = [4.0, 2.0, 6.0, 3.0]
    assert pick_level(lv, "low", 5.0) == 2.0
    assert pick_level(lv, "high", 5.0) == 6.0
    assert pick_level(lv, "mid", 5.0) == 3.0          # middle of the in-bank levels 2, 3, 4
    assert pick_level(lv, "mid", 1.0) == 4.0          # no in-bank level: middle of all
    assert pick_level(lv, 2.5, 5.0) == 2.5


def test_variant_reaches_one_base_per_level():
    sec = Section(B=12, Hb=3, z=0, Bf=0, n=0.03)
    cfg = ReachConfig(length=24, dx=0.5, cs=0.12)
    test = dict(key="T", title="t", variants=[
        dict(label="a", boat="longtail", rows=1, per_row=2, level="low"),
        dict(label="b", boat="outboard", rows=2, per_row=1, row_spacing=9.0, level="high", over=dict(tilt_deg=5)),
        dict(label="c", boat="tug", rows=1, per_row=1)])
    cases, bases = _variant_reaches(test, sec, [2.0, 3.0], 3.0, cfg,
                                    lambda h: (manning_discharge(sec, h, 3e-4), 3e-4), 6.0,
                                    {"tug": dict(power_kW=150)})
    assert sorted(bases) == [2.0, 3.0]
    assert [c[0] for c in cases] == [2.0, 3.0, 3.0]
    assert all(not b.fleet.enabled for b in bases.values())
    _, rb, _ = cases[1]
    assert rb.fleet.rows == 2 and rb.fleet.row_spacing == 9.0 and rb.fleet.boat.tilt_deg == 5
    assert cases[2][1].fleet.boat.power_kW == 150
    assert rb.fleet.x_first == 6.0


def test_run_to_end_steps_matches_the_run_loop():
    """batch.run_to_end_steps: the step count of Run3D.run_to_end's loop (400-step advance
    calls of 20-step chunks, t += 20 dt per chunk, until t >= t_total)."""
    from water_flow_simulation_b200.batch import run_to_end_steps
    from water_flow_simulation_b200.reach3d import Run3D, build_reach, Fleet, boat_type
    sec = Section(B=12, Hb=3, z=0, Bf=0, n=0.03)
    cfg = ReachConfig(length=24, dx=0.5, cs=0.12)
    r = build_reach(sec, 2.0, manning_discharge(sec, 2.0, 3e-4), 3e-4, Fleet(boat_type("tug"), enabled=False), cfg)
    t_total = cfg.run_flows * cfg.length / max(r.V, 0.05)
    t, steps = 0.0, 0
    while t < t_total:                 # Run3D.run_to_end -> advance(400) -> 20 chunks of 20
        for _ in range(20):
            t = t + 20 * r.dt
        steps += 400
    assert run_to_end_steps(r) == steps and steps % 400 == 0
    assert run_to_end_steps(r, chunk=20) >= t_total / r.dt
