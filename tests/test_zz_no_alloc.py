"""lbm_build_worklists_noalloc (static scratch) against lbm_build_worklists (caller scratch).

Collected last on purpose: it must give the same lists whether it runs in a fresh
process (its first call looks up the static array's device address) or after every
other test has used the library.  Each lattice is listed twice in a row into outputs
pre-filled with a sentinel, and two lattices alternate, so a stale byte left in the
shared static array from the previous call would show up as a wrong list.
"""
import ctypes

import numpy as np
import pytest

from golden_io import load_reach_case, load_step_case
from water_flow_simulation_b200 import _native as nat

NOALLOC_MAX_SEGMENTS = 4 << 20
LBM_ERR_ARG = -1
SENTINEL = -1


def _noalloc_lists(torch, L, v):
    lib = L.lib
    n = (L.pitch + 32 * v - 1) // (32 * v) * L.ny * L.nz
    lists = [torch.full((n,), SENTINEL, dtype=torch.int32, device=L.device) for _ in range(4)]
    counts = torch.full((4,), SENTINEL, dtype=torch.int32, device=L.device)
    rc = lib.lbm_build_worklists_noalloc(L._lattice_ref(), v, *(a.data_ptr() for a in lists), counts.data_ptr(),
                                         L._stream())
    nat.check(rc, "lbm_build_worklists_noalloc")
    torch.cuda.synchronize()
    return [a.cpu().numpy() for a in lists], tuple(int(x) for x in counts.cpu())


def _expected(L):
    lists, counts, v = L._wl
    return [a[:k].cpu().numpy() for a, k in zip(lists, counts)], counts, v


@pytest.mark.gpu
@pytest.mark.parametrize("tile", ((3, 2, 4, 0, 0), (3, 4, 4, 0, 0)))
def test_noalloc_lists_match_scratch_entry_point(tile):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from test_gpu_parity import make_solver
    solvers = [make_solver(load_step_case("mini_tug"), tile=tile), make_solver(load_reach_case("cfg1"), tile=tile),
               make_solver(load_step_case("mini_jet"), tile=tile, crop=33)]
    for _ in range(2):
        for L in solvers:
            want, want_counts, v = _expected(L)
            assert sum(want_counts) == (L.pitch + 32 * v - 1) // (32 * v) * L.ny * L.nz
            for _call in range(2):
                got, counts = _noalloc_lists(torch, L, v)
                assert counts == want_counts
                for g, w, k in zip(got, want, counts):
                    np.testing.assert_array_equal(g[:k], w)
                    assert np.all(g[k:] == SENTINEL)


def test_noalloc_rejects_lattices_over_the_static_limit():
    """nseg*ny*nz above 4194304 returns LBM_ERR_ARG before any device work (no GPU needed)."""
    import torch
    lib = nat.load()
    flags = torch.zeros(4, dtype=torch.int32)
    L = nat.Lattice()
    L.nx, L.ny, L.nz = 4096, 4096, 64
    L.pitch, L.cells = 4096, 4096 * 4096 * 64
    L.flags = L.uin = flags.data_ptr()
    outs = [flags.data_ptr()] * 5
    for v in (2, 4):
        n = 4096 // (32 * v) * 4096 * 64
        assert n > NOALLOC_MAX_SEGMENTS
        rc = lib.lbm_build_worklists_noalloc(ctypes.byref(L), v, *outs, None)
        assert rc == LBM_ERR_ARG
        msg = lib.lbm_last_error().decode()
        assert "4194304" in msg and "static limit" in msg, msg


@pytest.mark.parametrize("nx,ny,nz,v,accepted", (
    (64, 2048, 2048, 2, True),       # 1 segment per row x 4194304 rows: exactly the limit
    (128, 2048, 2048, 4, True),
    (320, 838861, 1, 2, False),      # 5 segments per row x 838861 rows = 4194305: one over
    (640, 838861, 1, 4, False),
))
def test_noalloc_limit_boundary(nx, ny, nz, v, accepted):
    """The segment limit is inclusive: 4194304 row segments pass the limit check (the call then
    stops at the NULL output arrays, before any device work) and 4194305 are refused."""
    import torch
    lib = nat.load()
    flags = torch.zeros(4, dtype=torch.int32)
    L = nat.Lattice()
    L.nx, L.ny, L.nz = nx, ny, nz
    L.pitch, L.cells = nx, nx * ny * nz
    L.flags = L.uin = flags.data_ptr()
    assert (nx // (32 * v)) * ny * nz == NOALLOC_MAX_SEGMENTS + (0 if accepted else 1)
    rc = lib.lbm_build_worklists_noalloc(ctypes.byref(L), v, None, None, None, None, None, None)
    assert rc == LBM_ERR_ARG
    msg = lib.lbm_last_error().decode()
    if accepted:
        assert "NULL array" in msg, msg
    else:
        assert "static limit" in msg and "4194305" in msg, msg
