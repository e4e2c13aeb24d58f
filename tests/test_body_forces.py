"""The force readout's definition on the CPU: the hull map of the reach builder, and the
oracle's momentum-exchange sum (oracle_body_forces_f32) on states whose answer is known."""
import numpy as np
import pytest

from oracle.oracle import OracleLBM, body_forces
from test_reach_builder import build_from_spec
from golden_io import load_step_case


@pytest.mark.parametrize("name", ("mini_tug", "mini_cfg1"))
def test_hull_map_is_the_carved_hull_cells(name):
    """body > 0 exactly where the boat's reach is solid and the no-boat reach is not, and each
    hull's cells lie inside its own box."""
    c = load_step_case(name)
    r = build_from_spec(c.spec)
    base = build_from_spec(dict(c.spec, fleet=dict(c.spec["fleet"], enabled=False)))
    assert r.body is not None and r.body.dtype == np.uint8 and base.body is None
    assert np.array_equal(r.body > 0, r.solid & ~base.solid)
    Xc = (np.arange(r.nx) + 0.5) * r.dx
    for k, (x0, x1, y0, y1, z0, _) in enumerate(r.hulls):
        z, y, x = np.nonzero(r.body == k + 1)
        assert len(x) > 0
        assert np.all((Xc[x] >= x0) & (Xc[x] <= x1) & (r.y[y] >= y0) & (r.y[y] <= y1) & (r.zc[z] >= z0))


def test_fluid_at_rest_exerts_no_net_force():
    """Populations at rest (f = w) around a cube in a closed box: the momentum exchange of every
    link is balanced by the opposite face's, so the net force is zero (and no body force)."""
    nz, ny, nx = 10, 12, 14
    solid = np.zeros((nz, ny, nx), bool)
    solid[:, :, 0] = solid[:, :, -1] = True
    body = np.zeros(solid.shape, np.uint8)
    body[3:7, 4:8, 5:9] = 1
    solid |= body > 0
    zero = np.zeros(solid.shape, np.float32)
    o = OracleLBM(solid, zero, zero, zero, np.zeros((nz, ny), np.float32), 0.6, 0.17)
    F = body_forces(o, body, 1)
    assert F.shape == (1, 3) and np.abs(F).max() < 1e-12


def test_uniform_pressure_difference_pushes_the_body():
    """Denser fluid upstream of a plate than downstream (f = rho w on each side): the force on
    the plate is along +x, of size (rho_up - rho_down)/3 x its cross-section (the lattice
    pressure rho/3 on each face), for plain bounce-back (no wall function)."""
    nz, ny, nx = 8, 8, 16
    solid = np.zeros((nz, ny, nx), bool)
    body = np.zeros(solid.shape, np.uint8)
    body[2:6, 2:6, 8] = 1
    solid |= body > 0
    zero = np.zeros(solid.shape, np.float32)
    o = OracleLBM(solid, zero, zero, zero, np.zeros((nz, ny), np.float32), 0.6, 0.17)
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)
    rho = np.where(np.arange(nx) < 8, np.float32(1.03), np.float32(1.0)).astype(np.float32)
    o.f = np.ascontiguousarray((w[:, None, None, None] * rho[None, None, None, :]
                                * np.ones((19, nz, ny, nx), np.float32)).ravel())
    F = body_forces(o, body, 1)[0]
    # every plate cell is the source of five links from each side (the axis one, w = 1/18, and
    # four diagonals, w = 1/36): 2 rho (1/18 + 4/36) = rho/3 per cell and side; the side faces'
    # links cancel in pairs
    assert abs(F[1]) < 1e-9 and abs(F[2]) < 1e-9
    want = 16 * (2 * (float(np.float32(1.03) * w[1]) + 4 * float(np.float32(1.03) * w[7]))
                 - 2 * (float(w[1]) + 4 * float(w[7])))
    assert abs(F[0] - want) < 1e-12 and abs(want - 16 * 0.03 / 3) < 1e-6
