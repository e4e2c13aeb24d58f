"""Warm-start network on the tensor cores against its CPU oracle (needs a B200).

The GPU path keeps weights, activations and back-propagated gradients in bf16 and accumulates
in float32; the oracle computes in float64 from the same bf16 weights and rounds to bf16 at the
same places (oracle.surrogate_oracle.bf16), so the two differ only by float32 accumulation
order and the rare bf16 tie it flips: forward output, loss and every layer's weight and bias
gradient agree to 1% in norm.  (Without the matched rounding, ReLU masks flipping on the tiny
half-resolution grids alone move those layers' gradients by several per cent.)
"""
import numpy as np
import pytest

from oracle.surrogate_oracle import bf16, forward_backward

pytestmark = pytest.mark.gpu


def _require_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("dims", ((2, 4, 6), (4, 6, 8)))
def test_forward_loss_and_gradients_match_oracle(dims):
    torch = _require_gpu()
    from water_flow_simulation_b200.surrogate import SurrogateNet
    net = SurrogateNet(seed=1)
    rng = np.random.default_rng(2)
    V = dims[0] * dims[1] * dims[2]
    x = rng.standard_normal((V, 8)).astype(np.float32)
    xb = torch.as_tensor(x).to(torch.bfloat16)
    target = rng.standard_normal((V, 4)).astype(np.float32)
    mask = (rng.random(V) > 0.25).astype(np.float32)
    net.zero_grad()
    loss, out = net.loss_and_grad(xb.cuda(), dims, torch.as_tensor(target), torch.as_tensor(mask))
    net.check()
    params = {k: (v["Wb"].float().cpu().numpy().astype(np.float64), v["b"].cpu().numpy().astype(np.float64))
              for k, v in net.p.items()}
    l_ref, out_ref, grads = forward_backward(params, xb.float().numpy().astype(np.float64), dims,
                                             target.astype(np.float64), mask.astype(np.float64), quant=bf16)
    errs = {k: (_rel(v["dW"].cpu().numpy(), grads[k][0]), _rel(v["db"].cpu().numpy(), grads[k][1]))
            for k, v in net.p.items()}
    print("forward", _rel(out.cpu().numpy(), out_ref), "loss", float(loss), l_ref, "grads", errs)
    assert _rel(out.cpu().numpy(), out_ref) < 0.01
    assert abs(float(loss) - l_ref) <= 0.01 * l_ref
    for k, (ew, eb) in errs.items():
        assert ew < 0.01 and eb < 0.01, (k, ew, eb)


def test_training_reduces_the_loss():
    torch = _require_gpu()
    from water_flow_simulation_b200.surrogate import SurrogateNet
    net = SurrogateNet(seed=3)
    rng = np.random.default_rng(4)
    dims = (4, 8, 12)
    V = 4 * 8 * 12
    x = torch.as_tensor(rng.standard_normal((V, 8)).astype(np.float32)).cuda()
    t = torch.as_tensor(np.tanh(rng.standard_normal((V, 4))).astype(np.float32)).cuda()
    m = torch.ones(V).cuda()
    first = None
    for _ in range(120):
        net.zero_grad()
        loss, _ = net.loss_and_grad(x, dims, t, m)
        net.adam(lr=2e-3)
        first = first if first is not None else float(loss)
    net.check()
    assert float(loss) < 0.5 * first


def test_lift_of_a_zero_prediction_is_the_1d_start():
    """A zero departure lifts to feq(1, (uin, 0, 0)): the reference's own start state."""
    torch = _require_gpu()
    import ctypes
    from water_flow_simulation_b200 import _native as nat
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.reach3d import Run3D
    from water_flow_simulation_b200.surrogate import FACTOR, N_OUT, RHO_SCALE, U_SCALE, coarse_dims
    run = Run3D(config1_case())
    L = run.lbm
    Z, Y, X = coarse_dims(L.nz, L.ny, L.nx)
    zero = torch.zeros(Z * Y * X, N_OUT, device=L.device)
    f = torch.empty(19 * L.cells, device=L.device)
    lat = L._lattice()
    nat.check(L.lib.lbm_lift_coarse(ctypes.byref(lat), zero.data_ptr(), N_OUT, X, Y, Z, FACTOR, U_SCALE, RHO_SCALE,
                                    f.data_ptr(), L._stream()), "lbm_lift_coarse")
    assert float((f - L.f).abs().max()) < 1e-7
