"""LBM_STEP_OVERLAP (needs a B200): the edge and special kernels on the library's side stream
beside the plain kernel give the same step, bit for bit, as the three kernels in order.

The kernels of one step read only the previous populations and write disjoint cells, so the
order in which they run cannot change a bit; the fork/join must still order every step after
the one before and the output-step kernels (solid fields, column means) after both parts.
"""
import numpy as np
import pytest

from golden_io import load_step_case
from test_gpu_fp16 import case as fp16_case
from test_gpu_parity import _require_gpu, make_solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ("long_channel", "mini_tug", "mini_jet"))
@pytest.mark.parametrize("storage,tile", (("fp16", (3, 2, 4, 0, 2)), ("fp16", (3, 2, 4, 0, 0)),
                                          ("fp32", (3, 4, 4, 0, 2)), ("fp32", (3, 2, 4, 0, 0))))
def test_overlap_is_bit_identical(name, storage, tile):
    torch = _require_gpu()
    c = fp16_case(name)
    a = make_solver(c, storage=storage, tile=tile)
    b = make_solver(c, storage=storage, tile=tile + (1,))
    assert b.overlap and not a.overlap
    for L in (a, b):
        L.enable_averaging()
        for n in (1, 3, 20, 20):
            L.step(n, accumulate=n == 20)
    torch.cuda.synchronize()
    assert torch.equal(a.f.view(torch.int16 if storage == "fp16" else torch.int32),
                       b.f.view(torch.int16 if storage == "fp16" else torch.int32))
    for k in ("_rho", "_ux", "_uy", "_uz", "_colU", "_avg"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k
    assert a.status() == 0 and b.status() == 0


def test_overlap_on_a_second_stream():
    """Steps enqueued on a non-default torch stream fork from and join back into that stream."""
    torch = _require_gpu()
    c = load_step_case("mini_tug")
    a = make_solver(c, storage="fp16", tile=(3, 2, 4, 0, 0))
    b = make_solver(c, storage="fp16", tile=(3, 2, 4, 0, 2, 1))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.step(7)
        got = b.ux.clone()
    a.step(7)
    s.synchronize()
    assert torch.equal(got, a.ux)
    assert np.array_equal(b.populations(), a.populations())
