"""The batched boat-test runner (boat_tests.run_test) on a B200: the same results as running
each case alone with the same storage, and the same stop as Run3D.run_to_end."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from water_flow_simulation_b200.geometry import Section, manning_discharge
    from water_flow_simulation_b200.reach3d import ReachConfig
    sec = Section(B=12, Hb=3, z=0, Bf=0, n=0.03)
    cfg = ReachConfig(length=24, dx=0.5, cs=0.12)
    test = dict(key="T", title="small", variants=[
        dict(label="long-tail x2 low", boat="longtail", rows=1, per_row=2, level="low"),
        dict(label="outboard x1 high", boat="outboard", rows=1, per_row=1, level="high"),
        dict(label="tug x1", boat="tug", rows=1, per_row=1)])
    return test, sec, [2.0, 3.0], 3.0, cfg, (lambda h: (manning_discharge(sec, h, 3e-4), 3e-4))


def test_batched_run_test_equals_case_by_case():
    from water_flow_simulation_b200.boat_tests import run_test
    test, sec, levels, h_sel, cfg, flow = _setup()
    seen = []
    batched = run_test(test, None, sec, levels, h_sel, cfg, None, flow, x_first=6.0,
                       on_result=lambda c, run: seen.append((c["label"], run.lbm.nstep)))
    single = run_test(test, None, sec, levels, h_sel, cfg, None, flow, x_first=6.0, batched=False)
    assert [c["label"] for c in batched] == [v["label"] for v in test["variants"]] == [s[0] for s in seen]
    for a, b in zip(batched, single):
        for key in ("profiles", "base_profiles"):
            for k, v in a[key].items():
                assert np.array_equal(v, b[key][k]), (a["label"], key, k)
        for k, v in a.items():
            if isinstance(v, float):
                assert v == b[k] or (v != v and b[k] != b[k]), (a["label"], k)


def test_batch_stops_where_run_to_end_stops():
    from water_flow_simulation_b200.batch import run_to_end_steps
    from water_flow_simulation_b200.boat_tests import _variant_reaches
    from water_flow_simulation_b200.reach3d import Run3D
    test, sec, levels, h_sel, cfg, flow = _setup()
    cases, _ = _variant_reaches(test, sec, levels, h_sel, cfg, flow, 6.0, None)
    r = cases[2][1]
    run = Run3D(r, storage="fp16")
    run.run_to_end()
    assert run.lbm.nstep == run_to_end_steps(r) and run.lbm.nstep % 400 == 0
