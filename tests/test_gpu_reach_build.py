"""The device reach builder (lbm_build_reach_masks / lbm_build_reach_walls,
reach_device.build_reach_device) against the host builder, array for array (needs a B200)."""
import numpy as np
import pytest

from golden_io import GOLDEN, REACH_CASES, Case
from test_reach_device import bumpy_args, spec_args

pytestmark = pytest.mark.gpu


def _compare(args, bumps):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from water_flow_simulation_b200.reach3d import build_reach
    from water_flow_simulation_b200.reach_device import build_reach_device, to_host
    ref = build_reach(*args, bed_bumps=bumps)
    dev = build_reach_device(*args, bed_bumps=bumps)
    assert dev.solid.is_cuda and dev.Fx.is_cuda
    got = to_host(dev)
    for k in ("solid", "Fx", "Fy", "Fz", "cf", "bedwall"):
        a, b = getattr(got, k), getattr(ref, k)
        if b is None:
            assert a is None
            continue
        assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b), k
    assert (dev.dt, dev.V, dev.nx, dev.ny, dev.nz) == (ref.dt, ref.V, ref.nx, ref.ny, ref.nz)
    return ref, dev


@pytest.mark.parametrize("name", REACH_CASES)
def test_device_builder_equals_host_builder(name):
    _compare(spec_args(Case(f"{GOLDEN}/reach_{name}.npz").spec), None)


def test_device_builder_bumpy_bed_and_fleet():
    _compare(*bumpy_args())


def test_device_built_reach_steps_like_host_built():
    """Run3D on the device-built reach: the same fields after 40 steps as on the host-built."""
    from water_flow_simulation_b200.reach3d import Run3D
    ref, dev = _compare(*bumpy_args())
    out = []
    for r in (ref, dev):
        run = Run3D(r, storage="fp16")
        run.advance(40)
        out.append([getattr(run.lbm, k).cpu().numpy() for k in ("rho", "ux", "uy", "uz")])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
