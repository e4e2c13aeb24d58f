"""16-bit population storage (lbm_fused_step_h) against the float32 path and the oracle (needs a B200).

The 16-bit store keeps fp16((f_i - w_i) * scale).  Collision and every other operation
run in float32 on the decoded values, so from the same (16-bit representable) state one
16-bit step must give the float32 step's populations rounded to fp16: the bar below is
one fp16 unit in the last place of the deviation f - w (2^-10 |f - w|, twice the rounding
error, leaving room for the float32 rounding of the deviation-form collision) plus 1e-7
absolute, and the macroscopic fields within 1e-5 (they are computed from the same decoded
inputs).  Over many steps the rounding accumulates; the drift test states it.
"""
import numpy as np
import pytest

from golden_io import STEP_CASES, load_reach_case, load_step_case
from parity_util import case_arrays, make_oracle, rel_u_error
from test_gpu_parity import _require_gpu, fields, make_solver

pytestmark = pytest.mark.gpu

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)
FP16_REL = 2.0 ** -10
ABS_SLACK = 1e-7
TOL_U = 1e-5
TOL_RHO = 1e-5


class ReachCase:
    """A built reach in the shape of a golden case (for make_solver / make_oracle)."""

    def __init__(self, r):
        self.solid, self.F, self.cf, self.bedwall = r.solid, (r.Fx, r.Fy, r.Fz), r.cf, r.bedwall
        self.uin_lb = (r.uin_phys / r.vel).astype(np.float32)
        self.tau0 = 0.5 + 3 * max(1e-6 * r.dt / r.dx ** 2, 2e-4)
        self.cs = r.cfg.cs
        self.d = {}
        self.N = r.solid.size


def long_channel():
    """Config-1 channel and boat, 160 m long: 640 x 50 x 12 cells, so rows hold plain 256-cell segments."""
    from water_flow_simulation_b200.geometry import Section
    from water_flow_simulation_b200.reach3d import BoatType, Fleet, ReachConfig, build_reach
    sec = Section(B=12, Hb=3, z=0, Bf=0, n=0.03)
    boat = BoatType("custom", "long-tail style", hull_L=10.0, hull_B=2.0, draft=0.8, n_props=1, prop_D=0.30,
                    prop_depth=0.35, tilt_deg=12, prop_x=2.5, prop_spacing=0, power_kW=75)
    fleet = Fleet(boat, rows=1, per_row=1, x_first=60.0)
    return ReachCase(build_reach(sec, 3.0, 0.8 * 36, 3e-4, fleet, ReachConfig(length=160, dx=0.25, cs=0.12)))


_LONG = None


def case(name):
    global _LONG
    if name == "long_channel":
        if _LONG is None:
            _LONG = long_channel()
        return _LONG
    if name == "cfg1":
        return load_reach_case("cfg1")
    return load_step_case(name)


CASES = ("long_channel", "cfg1") + STEP_CASES


def pitched(L, f_ref):
    """Reference-layout host populations (19*N) -> float32 device tensor in L's pitched layout."""
    import torch
    f = torch.as_tensor(f_ref.reshape(19, L.nz, L.ny, L.nx), device=L.device)
    out = torch.as_tensor(W, device=L.device).view(19, 1, 1, 1).expand(19, L.nz, L.ny, L.pitch).clone()
    out[..., :L.nx] = f
    return out.reshape(-1)


def dev_bound(f_ref):
    w = np.repeat(W, f_ref.size // 19)
    return FP16_REL * np.abs(f_ref - w) + ABS_SLACK


def test_case_has_plain_segments():
    _require_gpu()
    L = make_solver(case("long_channel"), storage="fp16")
    for tile in ((3, 2, 4, 0, 0), (3, 4, 4, 0, 0), (3, 8, 4, 0, 0)):
        L.set_tile(tile)
        plain, solid, special, edge = L.worklist_counts()
        assert plain > 0 and special > 0 and edge > 0, (tile, plain, solid, special, edge)


@pytest.mark.parametrize("name", CASES)
def test_start_state_decodes_to_float_start(name):
    _require_gpu()
    c = case(name)
    L16, L32 = make_solver(c, storage="fp16"), make_solver(c)
    f16, f32 = L16.populations(), L32.populations()
    w = np.repeat(W, f32.size // 19)
    assert np.all(np.abs(f16 - f32) <= 2.0 ** -11 * np.abs(f32 - w) + 1e-12)


@pytest.mark.parametrize("name", ("long_channel", "mini_tug"))
def test_pack_unpack(name):
    """decode(encode(f)) is f rounded (half an fp16 ulp of f - w).  encode(decode(h)) == h bit for bit
    wherever |f - w| >= 2^-12 (there w + d is exact in float32); below that the float32 sum w + d
    itself rounds, and re-encoding moves the population by at most one float32 ulp of w."""
    import torch
    _require_gpu()
    L = make_solver(case(name), storage="fp16")
    L.step(3)
    h0 = L.f.clone()
    f = L.populations_device()
    L.load_populations(f)
    d0 = h0.float() / L.store_scale
    big = d0.abs() >= 2.0 ** -12
    assert torch.equal(L.f.view(torch.int16)[big], h0.view(torch.int16)[big])
    f_again = L.populations_device()
    w_full = torch.as_tensor(np.repeat(W, L.cells), device=L.device)
    assert bool(((f_again - f).abs() <= 2.0 ** -11 * (f - w_full).abs() + 2.0 ** -25).all())
    rng = np.random.default_rng(5)
    g = (W[:, None] * (1 + 0.3 * rng.standard_normal((19, L.cells)))).astype(np.float32).ravel()
    L.load_populations(torch.as_tensor(g, device=L.device))
    back = L.populations_device().cpu().numpy()
    w = np.repeat(W, L.cells)
    assert np.all(np.abs(back - g) <= 2.0 ** -11 * np.abs(g - w) + 1e-12)


TILES16 = ((3, 2, 4, 0, 0), (3, 4, 4, 0, 0), (3, 8, 4, 0, 0), (3, 2, 1, 0, 0), (3, 2, 4, 4, 0), (3, 4, 2, 4, 0))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("crop", (None, 61, 57, 65))
@pytest.mark.parametrize("tile", TILES16)
def test_one_step_is_float_step_rounded(name, crop, tile):
    """From the same decoded state, a 16-bit step = the float32 step rounded to the 16-bit store.

    Where x = nx-1 starts a segment pass (nx-1 a multiple of 32 x cells per lane of the general
    path; crop 65 with 2 cells per lane) the outlet is extrapolated in a separate pass from the
    stored, rounded x = nx-2 populations g: the outlet then also carries their rounding,
    |d out_i| <= |d g_i| + w_i sum_j |d g_j|, each |d g_j| <= 2^-11 |g_j - w_j|."""
    _require_gpu()
    if crop is not None and name not in ("mini_tug", "long_channel"):
        pytest.skip("ragged crops on two geometries")
    c = case(name)
    if crop is not None and name == "long_channel":
        crop = 600 + crop % 8          # nx % 8 != 0 with plain segments present
    L16 = make_solver(c, storage="fp16", crop=crop, tile=tile)
    L32 = make_solver(c, crop=crop)
    L16.step(2)                                     # a non-trivial state (wall-function fields set)
    L32.load_populations(pitched(L32, L16.populations()))
    for a in ("_rho", "_ux", "_uy", "_uz"):
        src = getattr(L16, a).view(L16.nz, L16.ny, L16.pitch)[..., :L16.nx]
        getattr(L32, a).view(L32.nz, L32.ny, L32.pitch)[..., :L32.nx].copy_(src)
    L32._colU.view(L32.ny, L32.pitch)[:, :L32.nx].copy_(L16._colU.view(L16.ny, L16.pitch)[:, :L16.nx])
    L16.step(1)
    L32.step(1)
    f16, f32 = L16.populations(), L32.populations()
    fluid = np.tile(~case_arrays(c, crop)[0].ravel(), 19)
    bnd = dev_bound(f32).reshape(19, L16.nz, L16.ny, L16.nx)
    vg = 2 if tile[1] == 2 else 4
    if (L16.nx - 1) % (32 * vg) == 0:
        dg = np.abs(f32.reshape(bnd.shape)[..., -2] - W[:, None, None])
        bnd[..., -1] += FP16_REL * (dg + W[:, None, None] * dg.sum(0, keepdims=True))
    bnd = bnd.ravel()
    err = np.abs(f16 - f32)[fluid]
    assert np.all(err <= bnd[fluid]), float((err / bnd[fluid]).max())
    g16, g32 = fields(L16), fields(L32)
    assert rel_u_error(g16, g32) < TOL_U and float(np.abs(g16["rho"] - g32["rho"]).max()) < TOL_RHO
    assert L16.status() == 0


@pytest.mark.parametrize("name", ("long_channel", "cfg1", "mini_tug", "mini_jet"))
def test_one_step_vs_oracle(name):
    """The oracle stepped from the decoded 16-bit start state, vs one 16-bit step."""
    _require_gpu()
    c = case(name)
    L16 = make_solver(c, storage="fp16", column=False)
    O = make_oracle(c)
    O.f = L16.populations().astype(np.float32)
    L16.step(1)
    O.step(1)
    f16 = L16.populations()
    fluid = np.tile(~c.solid.ravel(), 19)
    bound = FP16_REL * np.abs(O.f - np.repeat(W, O.f.size // 19)) + 2 * ABS_SLACK
    err = np.abs(f16 - O.f)
    assert np.all(err[fluid] <= bound[fluid]), float((err[fluid] / bound[fluid]).max())
    g = fields(L16)
    assert rel_u_error(g, O) < TOL_U and float(np.abs(g["rho"] - O.rho).max()) < TOL_RHO


def test_rest_state_stays_exact():
    """A closed box at rest: the 16-bit deviations stay exactly zero (plain and general segments)."""
    import torch
    _require_gpu()
    from water_flow_simulation_b200.lbm3d import LBM3D
    nz, ny, nx = 8, 10, 600
    solid = np.zeros((nz, ny, nx), bool)
    solid[:, :, 0] = solid[:, :, -1] = True
    zero = np.zeros_like(solid, np.float32)
    L = LBM3D(None, solid, zero, zero, zero, np.zeros((nz, ny), np.float32), 0.52, 0.17, storage="fp16")
    assert L.worklist_counts()[0] > 0
    L.step(40)
    assert int(torch.count_nonzero(L.f)) == 0
    assert float(L.ux.abs().max()) == 0.0 and float((L.rho - 1).abs().max()) == 0.0


def test_rejects_bad_scale_and_tile():
    import torch
    _require_gpu()
    from water_flow_simulation_b200 import _native as nat
    L = make_solver(case("mini_tug"), storage="fp16")
    rc = L.lib.lbm_fused_step_h(L._lattice_ref(), L.f.data_ptr(), L.f2.data_ptr(), 3000.0, 1, L.tile, L._stream())
    assert rc == -1 and b"power of two" in L.lib.lbm_last_error()
    bad = nat.Tile(3, 3, 4, 0, 0)
    rc = L.lib.lbm_fused_step_h(L._lattice_ref(), L.f.data_ptr(), L.f2.data_ptr(), L.store_scale, 1, bad, L._stream())
    assert rc == -1 and b"2, 4 or 8 cells per lane" in L.lib.lbm_last_error()
    other = nat.Tile(3, 8, 4, 0, 0)                 # lists were built for 2 cells per lane
    rc = L.lib.lbm_fused_step_h(L._lattice_ref(), L.f.data_ptr(), L.f2.data_ptr(), L.store_scale, 1, other,
                                L._stream())
    assert rc == -1 and b"work lists" in L.lib.lbm_last_error()
    torch.cuda.synchronize()


def test_nan_sets_status_word():
    _require_gpu()
    c = case("long_channel")
    L = make_solver(c, storage="fp16")
    L.step(1)
    assert L.status() == 0
    i = int(np.flatnonzero(L._flags.cpu().numpy() == 0)[len(L._flags) // 3])
    L.f[i] = float("nan")
    L.step(1)
    assert L.status() & 1


@pytest.mark.parametrize("name", ("long_channel", "cfg1"))
def test_drift_against_float32_over_100_steps(name):
    """The accumulated 16-bit rounding after 100 steps against the float32 path, printed beside
    the float32 path's own sensitivity (the same 100 steps from a start state moved by one float32
    ulp per population), under a sanity bound (5% of max|u|, 1e-3 in density) that an encoding
    fault would exceed by orders of magnitude.  The field-level difference is dominated by the
    flow's own amplification of rounding, so the accuracy statement of the 16-bit store is made on
    water level and bed shear against the FP64 oracle instead."""
    import torch
    _require_gpu()
    c = case(name)
    L16, L32, L32p = make_solver(c, storage="fp16"), make_solver(c), make_solver(c)
    sgn = torch.as_tensor(np.random.default_rng(1).choice([-1.0, 1.0], L32p.f.numel()).astype(np.float32),
                          device=L32p.device)
    L32p.f.copy_(torch.nextafter(L32p.f, L32p.f + sgn))
    L32p.f2.copy_(L32p.f)
    for L in (L16, L32, L32p):
        L.step(100)
    g16, g32, g32p = fields(L16), fields(L32), fields(L32p)
    eu = rel_u_error(g16, g32)
    er = float(np.abs(g16["rho"] - g32["rho"]).max())
    spread = rel_u_error(g32p, g32)
    print(f"{name}: 100 steps, 16-bit vs float32: velocity {eu:.2e} of max|u|, density {er:.2e}; "
          f"float32 1-ulp spread {spread:.2e}")
    assert eu < 5e-2 and er < 1e-3, (eu, er)
