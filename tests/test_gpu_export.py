"""The device velocity export (lbm_export_velocity, export.export_case) against the
reference's own exports and the CPU oracle (needs a B200)."""
import json

import numpy as np
import pytest

from golden_io import GOLDEN
from test_export import EXPORT_CASES, _case
from test_reach_builder import build_from_spec

pytestmark = pytest.mark.gpu


def _run_with_sums(reach, sums, navg, storage):
    import torch
    from water_flow_simulation_b200.reach3d import Run3D
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    run = Run3D(reach, storage=storage)
    L = run.lbm
    L.enable_averaging()
    for k, s in enumerate(sums):
        dst = L._avg[k * L.cells:(k + 1) * L.cells].view(L.nz, L.ny, L.pitch)[..., :L.nx]
        dst.copy_(torch.from_numpy(np.asarray(s, np.float32).reshape(L.nz, L.ny, L.nx)))
    run.navg = L.navg = navg
    return run


@pytest.mark.parametrize("storage", ("fp32", "fp16"))
@pytest.mark.parametrize("name", EXPORT_CASES)
def test_device_export_equals_reference_export(name, storage):
    from water_flow_simulation_b200 import export
    c, sums, navg, res, ref = _case(name)
    reach = build_from_spec(c.spec)
    run = _run_with_sums(reach, sums, navg, storage)
    for _ in range(2):                                   # a second call sees the same result
        out = json.loads(json.dumps(export.export_case(run, "case", None, res)))
        assert out.pop("boat") == (reach.fleet.boat.name if reach.fleet.enabled else "")
        want = dict(ref)
        want.pop("boat")
        assert out == want


@pytest.mark.parametrize("seed", (0, 1))
def test_device_velocity_blocks_equal_oracle_on_config1(seed):
    """config-1 boat case (192 x 50 x 12) with seeded random sums, including exact ties of
    the int8 rounding and a block column of solids, against the oracle bit for bit."""
    from oracle.export_oracle import velocity_int8 as oracle_blocks
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.export import velocity_int8
    reach = config1_case()
    rng = np.random.default_rng(seed)
    N = reach.solid.size
    navg = 1 + seed * 40
    sums = [(navg * (0.1 + 0.05 * rng.standard_normal(N))).astype(np.float32) for _ in range(3)]
    run = _run_with_sums(reach, sums, navg, "fp32")
    q, scale, sp99 = velocity_int8(run)
    qo, so, spo = oracle_blocks(sums, navg, reach.vel, reach.solid)
    assert np.array_equal(q, qo)
    assert scale == so and sp99 == spo


def test_device_export_without_averages_uses_current_fields():
    """Run3D.field(mean=True) falls back to the current fields before any average: so does
    the export."""
    import torch
    from oracle.export_oracle import velocity_int8 as oracle_blocks
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.export import velocity_int8
    from water_flow_simulation_b200.reach3d import Run3D
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    reach = config1_case()
    run = Run3D(reach)
    run.advance(40)
    assert run.navg == 0
    fields = [getattr(run.lbm, k).cpu().numpy() for k in ("ux", "uy", "uz")]
    q, scale, sp99 = velocity_int8(run)
    qo, so, spo = oracle_blocks(fields, 1, reach.vel, reach.solid)
    assert np.array_equal(q, qo) and scale == so and sp99 == spo
