"""The CPU oracle of the warm-start network: its gradients against finite differences (CPU only)."""
import numpy as np

from oracle.surrogate_oracle import LAYERS, forward_backward


def _params(rng, scale=0.2):
    return {n: (rng.standard_normal((co, 27 * ci)) * scale / np.sqrt(27 * ci), rng.standard_normal(co) * 0.1)
            for n, ci, co, _ in LAYERS}


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = (2, 4, 4)
    V = 32
    params = _params(rng)
    x = rng.standard_normal((V, 8))
    target = rng.standard_normal((V, 4))
    mask = (rng.random(V) > 0.3).astype(float)
    loss, _, grads = forward_backward(params, x, dims, target, mask)
    eps = 1e-6
    for name in ("c1", "c3", "c6"):
        W, b = params[name]
        for idx in [(0, 0), (W.shape[0] - 1, W.shape[1] - 1), (W.shape[0] // 2, W.shape[1] // 3)]:
            Wp = W.copy()
            Wp[idx] += eps
            lp = forward_backward({**params, name: (Wp, b)}, x, dims, target, mask)[0]
            Wm = W.copy()
            Wm[idx] -= eps
            lm = forward_backward({**params, name: (Wm, b)}, x, dims, target, mask)[0]
            num = (lp - lm) / (2 * eps)
            assert abs(num - grads[name][0][idx]) <= 1e-6 + 1e-4 * abs(num), (name, idx, num, grads[name][0][idx])
        bp = b.copy()
        bp[0] += eps
        bm = b.copy()
        bm[0] -= eps
        num = (forward_backward({**params, name: (W, bp)}, x, dims, target, mask)[0]
               - forward_backward({**params, name: (W, bm)}, x, dims, target, mask)[0]) / (2 * eps)
        assert abs(num - grads[name][1][0]) <= 1e-6 + 1e-4 * abs(num)
