"""Parity on the benchmark geometries (needs a B200).

The bench steps the 36.1M-cell reach of cases.config2_case (a seeded bumpy bed, so the bed
height, the friction and the bed/bank mask vary along x, and a 20 m tug with two 300 kW
propellers) and the seeded cases of cases.ensemble_case.  Their flag words, wall-function
cells and work-list mix differ from the extruded-section golden cases, so they are stepped
here against the oracle too:

* reach36m_tug_window -- columns 380..619 of the 1500 x 602 x 40 lattice itself (dx 0.1 m):
  the tug's hull and both propellers, the bumpy bed and the banks at full resolution,
  240 x 602 x 40 = 5.8M cells;
* reach36m_dx04 -- the whole 150 m reach with the same bed field and tug at dx 0.4 m
  (375 x 152 x 10): inlet, outlet and every part of the bed in one lattice;
* ensemble1 / ensemble12 -- two seeded ensemble cases at their benchmark size (an outboard
  boat at a 3 m stage, 100 bar jets at 4 m; 2.8M and 3.1M cells).

Bars: float32 fields after N = 1, 2, 5 steps within 1e-5 of max|u| (velocity) and 1e-5
absolute (density) of the oracle, or twice the oracle's own 1-ulp spread on that case where
that is larger (tests/parity_util.py), through the float32 default tile and the bench's
tile; the 16-bit store: one step equals the float32 step rounded to the store
(tests/test_gpu_fp16.py states that bar).
"""
import numpy as np
import pytest

from parity_util import case_arrays, case_bound, make_oracle
from test_gpu_fp16 import ReachCase, W, dev_bound, pitched
from test_gpu_parity import _require_gpu, errors, fields, make_solver

pytestmark = pytest.mark.gpu

TOL_U = 1e-5
TOL_RHO = 1e-5
NAMES = ("reach36m_tug_window", "reach36m_dx04", "ensemble1", "ensemble12")
# float32 default (16-byte accesses, 4 cells per lane) and the bench's 16-bit tile run in float32
TILES32 = ((3, 4, 4, 0, 0), (3, 2, 4, 0, 0))
_CASES = {}


class WindowCase(ReachCase):
    """Columns [x0, x1) of a built reach as a case of its own (inlet at x0, outlet at x1 - 1)."""

    def __init__(self, r, x0, x1):
        super().__init__(r)
        sl = (slice(None), slice(None), slice(x0, x1))
        self.solid = np.ascontiguousarray(r.solid[sl])
        self.F = tuple(np.ascontiguousarray(a[sl]) for a in (r.Fx, r.Fy, r.Fz))
        self.cf = None if r.cf is None else np.ascontiguousarray(r.cf[sl])
        self.bedwall = None if r.bedwall is None else np.ascontiguousarray(r.bedwall[sl])
        self.N = self.solid.size


def bench_case(name):
    if name not in _CASES:
        from water_flow_simulation_b200.cases import config2_case, ensemble_case
        if name == "reach36m_tug_window":
            _CASES[name] = WindowCase(config2_case(), 380, 620)
        elif name == "reach36m_dx04":
            _CASES[name] = ReachCase(config2_case(dx=0.4))
        else:
            _CASES[name] = ReachCase(ensemble_case(int(name[len("ensemble"):])))
    return _CASES[name]


@pytest.mark.parametrize("name", NAMES)
def test_geometry_has_every_segment_class(name):
    """The lattice carries plain, special (bed, banks, hull, propellers) and edge row segments,
    and propeller forcing, as the benchmark lattice does."""
    _require_gpu()
    c = bench_case(name)
    assert any(np.any(a != 0) for a in c.F) and c.bedwall is not None and c.bedwall.any()
    L = make_solver(c, tile=(3, 2, 4, 0, 0), storage="fp16")
    plain, solid, special, edge = L.worklist_counts()
    assert plain > 0 and special > 0 and edge > 0, (plain, solid, special, edge)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("tile", TILES32)
def test_fp32_vs_oracle(name, tile):
    _require_gpu()
    c = bench_case(name)
    L = make_solver(c, tile=tile)
    O = make_oracle(c)
    done = 0
    for n in (1, 2, 5):
        O.update_uref(c.bedwall)
        O.step(n - done)
        L.step(n - done)
        done = n
        eu, er = errors(L, O)
        assert eu < case_bound(name, c, n, TOL_U) and er < TOL_RHO, (name, tile, n, eu, er)
    assert L.status() == 0


@pytest.mark.parametrize("name", NAMES)
def test_fp16_one_step_is_float_step_rounded(name):
    """The bench's 16-bit tile: from the same decoded state, one 16-bit step equals the float32
    step rounded to the store (2^-10 |f - w| + 1e-7, plus the outlet's neighbour rounding
    where x = nx-1 starts a pass of its own), and the fields agree within 1e-5."""
    _require_gpu()
    c = bench_case(name)
    L16 = make_solver(c, storage="fp16", tile=(3, 2, 4, 0, 0))
    L32 = make_solver(c)
    L16.step(2)
    L32.load_populations(pitched(L32, L16.populations()))
    for a in ("_rho", "_ux", "_uy", "_uz"):
        src = getattr(L16, a).view(L16.nz, L16.ny, L16.pitch)[..., :L16.nx]
        getattr(L32, a).view(L32.nz, L32.ny, L32.pitch)[..., :L32.nx].copy_(src)
    L32._colU.view(L32.ny, L32.pitch)[:, :L32.nx].copy_(L16._colU.view(L16.ny, L16.pitch)[:, :L16.nx])
    L16.step(1)
    L32.step(1)
    f16, f32 = L16.populations(), L32.populations()
    fluid = np.tile(~case_arrays(c)[0].ravel(), 19)
    bnd = dev_bound(f32).reshape(19, L16.nz, L16.ny, L16.nx)
    if (L16.nx - 1) % 64 == 0:
        dg = np.abs(f32.reshape(bnd.shape)[..., -2] - W[:, None, None])
        bnd[..., -1] += 2.0 ** -10 * (dg + W[:, None, None] * dg.sum(0, keepdims=True))
    bnd = bnd.ravel()
    err = np.abs(f16 - f32)[fluid]
    assert np.all(err <= bnd[fluid]), float((err / bnd[fluid]).max())
    g16, g32 = fields(L16), fields(L32)
    umax = max(float(np.abs(g32[k]).max()) for k in ("ux", "uy", "uz"))
    eu = max(float(np.abs(g16[k] - g32[k]).max()) for k in ("ux", "uy", "uz")) / umax
    assert eu < TOL_U and float(np.abs(g16["rho"] - g32["rho"]).max()) < TOL_RHO
    assert L16.status() == 0
