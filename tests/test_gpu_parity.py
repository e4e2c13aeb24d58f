"""CUDA path vs the CPU oracle and the reference's golden outputs (needs a B200).

Bars:
* bit for bit: the flag maps (wall mask, solid, force, wall-function and bed/bank
  bits) and the initial populations;
* FP32 fields: after N <= 5 steps, velocity within TOL_U = 1e-5 of max|u|
  (max-norm) and density within TOL_RHO = 1e-5 absolute, of the reference's own
  Numba outputs (golden fixtures) and of the oracle.  Where the reference path
  itself is less stable than that -- the wall function normalises a tangential
  velocity that can be tiny, so one float32 ulp in its start state already moves
  the fields by more than 1e-5 after a few steps -- the bar is twice that measured
  1-ulp spread of the reference path (tests/parity_util.py).  Config 1, the
  case the 1e-5 figure is quoted on, stays inside 1e-5 itself.
"""
import numpy as np
import pytest

from golden_io import STEP_CASES, load_reach_case, load_step_case
from oracle.oracle import equilibrium_init, wall_mask
from parity_util import bound, case_arrays, make_oracle, oracle_spread, rel_u_error

pytestmark = pytest.mark.gpu

TOL_U = 1e-5
TOL_RHO = 1e-5
# (pipeline, cells_per_lane, warps, stages, ctas_per_sm): TMA-staged and register/shuffle pipelines
TILES = [(3, 4, 4, 0, 0), (3, 2, 4, 0, 0), (2, 2, 4, 3, 0), (1, 1, 4, 4, 0), (0, 2, 4, 0, 0), (0, 4, 4, 0, 0),
         (1, 1, 8, 3, 0), (2, 2, 1, 2, 0), (2, 2, 8, 4, 0), (1, 1, 2, 2, 0), (3, 4, 1, 0, 0)]


def _require_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def make_solver(c, tile=None, column=True, crop=None, **kw):
    from water_flow_simulation_b200.lbm3d import LBM3D
    solid, F, cf, bw = case_arrays(c, crop)
    use_col = column and bw is not None
    L = LBM3D(None, solid, *F, c.uin_lb, c.tau0, c.cs, cf, bedwall=bw if use_col else None,
              uref_mode="column" if use_col else "field", tile=tile, **kw)
    if "csmag2" in c.d:
        L.csmag2 = float(c.d["csmag2"])
    return L


def fields(L):
    return {k: getattr(L, k).cpu().numpy() for k in ("rho", "ux", "uy", "uz")}


def errors(L, ref):
    g = fields(L)
    r = ref if isinstance(ref, dict) else {k: getattr(ref, k) for k in ("rho", "ux", "uy", "uz")}
    return rel_u_error(g, r), float(np.abs(g["rho"] - r["rho"]).max())


def expected_wallfn(solid, cf):
    """Cells where floodsim/lbm3d.py:68-74 enters the wall function: cf > 0, a wall
    in the mask, a non-zero summed wall normal and a non-zero face area."""
    from oracle.oracle import CX, CY, CZ
    wm = wall_mask(solid)
    bit = lambda i: ((wm >> np.uint32(i)) & 1).astype(np.int64)  # noqa: E731
    nx_ = sum(-CX[i] * bit(i) for i in range(1, 19))
    ny_ = sum(-CY[i] * bit(i) for i in range(1, 19))
    nz_ = sum(-CZ[i] * bit(i) for i in range(1, 19))
    area = (bit(1) + bit(2)) ** 2 + (bit(3) + bit(4)) ** 2 + (bit(5) + bit(6)) ** 2
    return (cf > 0) & (wm != 0) & (nx_ ** 2 + ny_ ** 2 + nz_ ** 2 > 0) & (area > 0) & ~solid


@pytest.mark.parametrize("name", STEP_CASES)
def test_initial_populations_bit_exact(name):
    _require_gpu()
    c = load_step_case(name)
    L = make_solver(c)
    assert np.array_equal(L.populations(), equilibrium_init(c.solid, c.uin_lb))


@pytest.mark.parametrize("name", ("cfg1", "tug_trap", "jet_flood", "curtain_nowm", "shallow_outboard", "base_rect"))
def test_flag_maps_bit_exact(name):
    _require_gpu()
    from water_flow_simulation_b200 import _native as nat
    c = load_reach_case(name)
    L = make_solver(c)
    fl = L.flags.cpu().numpy().astype(np.uint32).reshape(c.shape)
    assert np.array_equal(fl & nat.FLAG_WALLS, wall_mask(c.solid))
    assert np.array_equal((fl & nat.FLAG_SOLID) != 0, c.solid)
    force = (c.F[0] != 0) | (c.F[1] != 0) | (c.F[2] != 0)
    assert np.array_equal((fl & nat.FLAG_FORCE) != 0, force & ~c.solid)
    if c.bedwall is not None:
        assert np.array_equal((fl & nat.FLAG_BEDWALL) != 0, c.bedwall & ~c.solid)
        assert np.array_equal((fl & nat.FLAG_WALLFN) != 0, expected_wallfn(c.solid, c.cf))


@pytest.mark.parametrize("name", STEP_CASES)
@pytest.mark.parametrize("tile", TILES[:6])
def test_fused_matches_reference_outputs(name, tile):
    """The reference's own Numba states (golden) after 1, 2 and 5 steps, uref cadence as Run3D."""
    _require_gpu()
    c = load_step_case(name)
    L = make_solver(c, tile=tile)
    done = 0
    for n in (1, 2, 5):
        L.step(n - done)
        done = n
        eu, er = errors(L, c.state(n))
        assert eu < bound(c, n, TOL_U) and er < TOL_RHO, (name, n, eu, er, oracle_spread(c, n)[n - 1])
    assert L.status() == 0


def test_config1_mini_within_1e5_for_5_steps():
    """On the config-1 physics the plain 1e-5 bar holds (no spread allowance)."""
    _require_gpu()
    c = load_step_case("mini_cfg1")
    L = make_solver(c)
    L.step(1)
    L.step(1)
    L.step(3)
    eu, er = errors(L, c.state(5))
    assert eu < TOL_U and er < TOL_RHO, (eu, er)


@pytest.mark.parametrize("name", ("mini_cfg1", "mini_nowm"))
def test_fused_uref_cadence_25_steps(name):
    """25 steps in chunks 1,1,3,20: the fused column-mean refresh reproduces Run3D's uref cadence."""
    _require_gpu()
    c = load_step_case(name)
    L = make_solver(c)
    done = 0
    for n in (1, 2, 5, 25):
        L.step(n - done)
        done = n
    eu, er = errors(L, c.state(25))
    assert eu < bound(c, 25, 1e-4) and er < 1e-5, (eu, er)


@pytest.mark.parametrize("tile", TILES)
def test_fused_vs_oracle_config1_full_size(tile):
    """Config-1 lattice (192x50x12, wall model on, full forcing) vs the oracle, N = 1, 2, 5: 1e-5."""
    _require_gpu()
    c = load_reach_case("cfg1")
    L = make_solver(c, tile=tile)
    O = make_oracle(c)
    done = 0
    for n in (1, 2, 5):
        O.update_uref(c.bedwall)
        O.step(n - done)
        L.step(n - done)
        done = n
        eu, er = errors(L, O)
        assert eu < TOL_U and er < TOL_RHO, (tile, n, eu, er)


@pytest.mark.parametrize("crop", (61, 62, 63, 64, 57, 33))
@pytest.mark.parametrize("tile", ((3, 4, 4, 0, 0), (3, 2, 2, 0, 0), (0, 2, 4, 0, 0), (0, 4, 4, 0, 0), (1, 1, 4, 4, 0), (1, 1, 2, 3, 0),
                                  (2, 2, 4, 3, 0), (2, 2, 2, 2, 0)))
def test_ragged_nx_padding_and_outlet(crop, tile):
    """nx not a multiple of 4 (pitched layout, ghost cells) and nx % V == 1 (outlet in its own pass)."""
    _require_gpu()
    c = load_step_case("mini_tug")
    L = make_solver(c, tile=tile, crop=crop)
    O = make_oracle(c, crop=crop)
    _, _, _, bw = case_arrays(c, crop)
    for _ in range(3):
        O.update_uref(bw)
        O.step(1)
        L.step(1)
    eu, er = errors(L, O)
    assert eu < bound(c, 3, TOL_U, crop=crop) and er < TOL_RHO, (crop, tile, eu, er)
    fl = np.tile(~L._solid_np.ravel(), 19)
    assert np.abs(L.populations()[fl] - O.f[fl]).max() < 1e-5


@pytest.mark.parametrize("name", STEP_CASES)
def test_reference_abi_kernels_vs_oracle(name):
    """lbm_step/lbm_bc with the reference's own argument lists and layout, vs the oracle (5 steps)."""
    torch = _require_gpu()
    from water_flow_simulation_b200 import _native as nat
    lib = nat.load()
    c = load_step_case(name)
    O = make_oracle(c)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(np.ascontiguousarray(a).ravel(), device=dev)  # noqa: E731
    f, f2 = T(O.f.copy()), T(O.f.copy())
    solid = T(c.solid.astype(np.uint8))
    F = [T(a) for a in c.F]
    cf = T(c.cf if c.cf is not None else np.zeros(c.shape, np.float32))
    rho, ux, uy, uz = T(O.rho.copy()), T(O.ux.copy()), T(O.uy.copy()), T(O.uz.copy())
    uref = T(O.uref.copy())
    uin = T(c.uin_lb)
    p = lambda t: t.data_ptr()  # noqa: E731
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(5):
        if c.bedwall is not None:
            O.update_uref(c.bedwall)
            uref.copy_(T(O.uref))
        O.step(1)
        nat.check(lib.lbm_step(p(f), p(f2), p(solid), *(p(a) for a in F), p(rho), p(ux), p(uy), p(uz), p(cf),
                               p(uref), c.nx, c.ny, c.nz, c.tau0, O.csmag2, st), "lbm_step")
        nat.check(lib.lbm_bc(p(f2), p(solid), p(uin), c.nx, c.ny, c.nz, 1.0, st), "lbm_bc")
        f, f2 = f2, f
    torch.cuda.synchronize()
    got = {"rho": rho.cpu().numpy(), "ux": ux.cpu().numpy(), "uy": uy.cpu().numpy(), "uz": uz.cpu().numpy()}
    eu = rel_u_error(got, O)
    er = float(np.abs(got["rho"] - O.rho).max())
    assert eu < bound(c, 5, TOL_U) and er < TOL_RHO, (eu, er)


def test_closed_box_mass_and_rest_state():
    """A box walled on all six sides: at rest it stays at rest; with forcing, the density sum
    drifts exactly as the reference's does (its float32 weights sum to 1 + 1.49e-8)."""
    torch = _require_gpu()
    from oracle.oracle import OracleLBM
    from water_flow_simulation_b200.lbm3d import LBM3D
    nz, ny, nx = 10, 20, 40
    solid = np.zeros((nz, ny, nx), bool)
    solid[:, :, 0] = solid[:, :, -1] = True
    zero = np.zeros_like(solid, np.float32)
    uin = np.zeros((nz, ny), np.float32)
    L = LBM3D(None, solid, zero, zero, zero, uin, 0.52, 0.17)
    L.step(50)
    assert float(L.ux.abs().max()) == 0.0 and float(L.uz.abs().max()) == 0.0
    Fx = zero.copy()
    Fx[3:7, 5:15, 10:30] = 1e-5
    L2 = LBM3D(None, solid, Fx, zero, zero, uin, 0.52, 0.17)
    O = OracleLBM(solid, Fx, zero, zero, uin, 0.52, 0.17)
    fluid = ~solid.ravel()
    m0 = float(O.rho[fluid].astype(np.float64).sum())
    L2.step(200)
    O.step(200)
    dm_gpu = float(L2.rho.cpu().numpy()[fluid].astype(np.float64).sum()) - m0
    dm_ref = float(O.rho[fluid].astype(np.float64).sum()) - m0
    assert abs(dm_gpu - dm_ref) < 0.1 * abs(dm_ref) + 1e-7 * m0, (dm_gpu, dm_ref)
    assert float(L2.ux.max()) > 0


def test_type_errors_like_reference():
    """floodsim/lbm3d.py:392-394: wrong dtype or size raises TypeError at step()."""
    torch = _require_gpu()
    c = load_step_case("mini_cfg1")
    L = make_solver(c)
    L.Fx = torch.zeros(c.N, dtype=torch.float64, device=L.device)
    with pytest.raises(TypeError):
        L.step(1)
    L.Fx = torch.zeros(c.N, dtype=torch.float32, device=L.device)
    L.uref = np.zeros(c.N - 1, np.float32)
    with pytest.raises(TypeError):
        L.step(1)


def test_nan_sets_status_word():
    """A non-finite population (written from the host side) sets the device status bit."""
    _require_gpu()
    c = load_step_case("mini_cfg1")
    L = make_solver(c)
    L.step(1)
    assert L.status() == 0
    i = int(np.flatnonzero(~c.solid.ravel())[100])
    L.f[i] = float("nan")
    L.step(1)
    assert L.status() & 1


@pytest.mark.parametrize("crop", (61, 64))
def test_layer_views_equal_the_flat_fields(crop):
    """LBM3D.layer(name, z) is layer z of the flat reference-layout field (pitched and unpitched
    lattices), as a view: no copy of the field is made."""
    torch = _require_gpu()
    c = load_step_case("mini_tug")
    L = make_solver(c, crop=crop)
    L.step(2)
    for name in ("rho", "ux", "uy", "uz"):
        full = getattr(L, name).view(L.nz, L.ny, L.nx)
        for z in (0, L.nz // 2, -1):
            lay = L.layer(name, z)
            assert lay.shape == (L.ny, L.nx) and torch.equal(lay, full[z]), (name, z)
            assert lay.untyped_storage().data_ptr() == getattr(L, "_" + name).untyped_storage().data_ptr()
    with pytest.raises(ValueError):
        L.layer("f")
