"""The host part of the device reach builder (reach_device.plan_reach) on the CPU: the
columns, hull segments and sparse forces it hands to the device describe exactly the host
builder's arrays, and its scalars, inlet profile and boats are the host builder's."""
from dataclasses import replace

import numpy as np
import pytest

from golden_io import GOLDEN, REACH_CASES, Case
from water_flow_simulation_b200.geometry import Section
from water_flow_simulation_b200.reach3d import BoatType, Fleet, ReachConfig, boat_type, build_reach, wall_cf


def spec_args(spec):
    key, over = spec["boat"]
    b = BoatType("custom", **over) if key == "custom" else replace(boat_type(key), **over)
    return (Section(**spec["sec"]), spec["h"], spec["Q"], spec["S"], Fleet(b, **spec["fleet"]),
            ReachConfig(**spec["cfg"]))


def bumpy_args():
    from water_flow_simulation_b200.cases import gaussian_bumps
    from water_flow_simulation_b200.geometry import manning_discharge
    sec = Section(B=14.0, Hb=3.0, z=2.0, Bf=0.0, n=0.025)
    tug = replace(boat_type("tug"), hull_L=8.0, hull_B=3.0, draft=1.0, prop_spacing=1.5)
    fleet = Fleet(tug, rows=2, per_row=2, row_spacing=12.0, x_first=6.0)
    return (sec, 3.0, manning_discharge(sec, 3.0, 3e-4), 3e-4, fleet, ReachConfig(length=40.0, dx=0.25, cs=0.17)), \
        gaussian_bumps(0.15, 2.0, 5)


def dense_from_plan(P):
    from water_flow_simulation_b200.reach_device import _ColumnSolid
    nz, ny, nx = P.nz, P.ny, P.nx
    z = np.arange(nz)[:, None, None]
    bed = (z < P.kb[None]) | P.outside[None, :, None]
    solid = bed.copy()
    for x in range(nx):
        for k in range(P.seg_off[x], P.seg_off[x + 1]):
            y0, y1, z0 = P.segs[k]
            solid[z0:, y0:y1 + 1, x] = True
    F = []
    for vals in P.F:
        a = np.zeros(nz * ny * nx, np.float32)
        a[P.keys] = vals
        F.append((a * P.k).astype(np.float32).reshape(nz, ny, nx))
    return solid, bed, F


CASES = [("golden", n) for n in REACH_CASES] + [("bumpy", None)]


@pytest.mark.parametrize("kind,name", CASES)
def test_plan_describes_host_arrays(kind, name):
    from water_flow_simulation_b200.reach_device import plan_reach
    if kind == "golden":
        args, bumps = spec_args(Case(f"{GOLDEN}/reach_{name}.npz").spec), None
    else:
        args, bumps = bumpy_args()
    ref = build_reach(*args, bed_bumps=bumps)
    P = plan_reach(*args, bed_bumps=bumps)
    solid, bed, F = dense_from_plan(P)
    assert np.array_equal(solid, ref.solid)
    for a, b in zip(F, (ref.Fx, ref.Fy, ref.Fz)):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    assert (P.dt, P.V, P.A, P.W, P.dx) == (ref.dt, ref.V, ref.A, ref.W, ref.dx)
    assert np.array_equal(P.uin, ref.uin_phys) and P.hulls == ref.hulls and P.notes == ref.notes
    assert [sorted(p.items()) for p in P.props] == [sorted(p.items()) for p in ref.props]
    if ref.cf is not None:
        cf, bw = wall_cf(solid, bed, P.dx, args[0].n, args[5])
        assert np.array_equal(cf, ref.cf) and np.array_equal(bw, ref.bedwall)
        cf_col = P.cf_col
        assert np.array_equal(ref.cf[ref.bedwall], np.broadcast_to(cf_col[None], ref.cf.shape)[ref.bedwall])


def test_benchmark_case_grids():
    """The benchmark cases' lattices follow the reference's grid rule (nz = round(h/dx), dx
    then h/nz, nx = round(L/dx), ny = ceil(W/dx) + 2): config 3 at a coarse dx that divides
    the 3.6 m stage (0.45 m), built; its full size at 0.05 m through the same grid rule, which
    build_reach calls, without allocating the 259.6M-cell lattice."""
    import math
    from water_flow_simulation_b200.cases import config3_case, config3_inputs, ensemble_case
    from water_flow_simulation_b200.reach3d import lattice_grid
    r = config3_case(dx=0.45)
    assert (r.nx, r.ny, r.nz) == (round(150 / 0.45), math.ceil(60 / 0.45) + 2, 8)
    sec, h, _, _, _, cfg, _ = config3_inputs(dx=0.45)
    assert lattice_grid(sec, h, cfg)[3:] == (r.nx, r.ny, r.nz) and lattice_grid(sec, h, cfg)[2] == r.dx
    sec, h, _, _, _, cfg, _ = config3_inputs()
    fp, W, dx, nx, ny, nz = lattice_grid(sec, h, cfg)
    assert (nx, ny, nz) == (3000, 1202, 72) and W == 60.0 and fp == 0.0
    assert nx * ny * nz == 259_632_000
    e = ensemble_case(0)
    assert 2.0e6 <= e.solid.size <= 2.0e7 * 1.2 and e.dx == 0.1
