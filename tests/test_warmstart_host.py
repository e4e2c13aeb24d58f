"""Host side of the learned warm start on the CPU: the coarse grid, the network's input
features and training targets (block means over 4 x 4 x 4 cells), the target scale, and the
seeded training cases."""
import numpy as np

from water_flow_simulation_b200.surrogate import (FACTOR, N_IN, N_PRED, RHO_SCALE, U_SCALE, case_features,
                                                  case_targets, coarse_dims)
from water_flow_simulation_b200.warmstart import random_case, target_scale


def test_coarse_dims_cover_the_lattice_with_even_counts():
    for n in ((12, 50, 192), (7, 9, 33), (40, 602, 1500)):
        d = coarse_dims(*n)
        assert all(c % 2 == 0 and c * FACTOR >= m for c, m in zip(d, n))
        assert all((c - 2) * FACTOR < m for c, m in zip(d, n))


def test_features_and_targets_are_block_means():
    rng = np.random.default_rng(0)
    nz, ny, nx = 8, 12, 16
    solid = np.zeros((nz, ny, nx), bool)
    solid[:2] = True                                            # a two-layer bed
    uin = rng.uniform(0.01, 0.05, (nz, ny)).astype(np.float32)
    F = [np.zeros((nz, ny, nx), np.float32) for _ in range(3)]
    x, dims = case_features(solid, *F, uin)
    assert x.shape == (np.prod(dims), N_IN) and x.dtype == np.float32
    Z, Y, X = dims
    feat = x.T.reshape(N_IN, Z, Y, X)
    # fluid fraction of the blocks: half the bottom block row is bed; y blocks past ny = 12 are padding
    assert np.allclose(feat[0, 0, :3], 0.5) and np.allclose(feat[0, 1, :3], 1.0) and np.all(feat[0, :, 3] == 0)
    rho = np.ones((nz, ny, nx)) + 1e-3
    ux = np.broadcast_to(uin[:, :, None], (nz, ny, nx)) + 0.01
    t, m = case_targets(solid, uin, rho, ux, np.zeros_like(rho), np.zeros_like(rho))
    assert t.shape == (np.prod(dims), N_PRED) and m.shape == (np.prod(dims),)
    assert np.allclose(t[m > 0, 0], 0.01 / U_SCALE, atol=1e-6)                # du over fluid cells only
    assert np.allclose(t[m > 0, 3], 1e-3 / RHO_SCALE, atol=1e-6)


def test_target_scale_is_the_masked_rms():
    t = np.array([[1.0, 2.0, 0.0, 4.0], [3.0, 2.0, 0.0, 0.0]], np.float32)
    m = np.array([1.0, 0.0], np.float32)
    s = target_scale([(None, None, t, m)])
    assert np.allclose(s, [1.0, 2.0, 0.0, 4.0], atol=1e-5)


def test_random_cases_are_seeded():
    a, b, c = random_case(3), random_case(3), random_case(4)
    assert np.array_equal(a.solid, b.solid) and a.dt == b.dt and a.props == b.props
    assert a.solid.shape != c.solid.shape or not np.array_equal(a.solid, c.solid)
