"""The optional outlet sponge (lbm_lattice.sponge_cols / sponge_tau; not in the reference)
against the CPU oracle with the same per-column relaxation time (needs a B200).

With sponge_cols = 0 every path is the reference's (all other tests); with a sponge the split
pipeline's special segments collide the last columns with tau0 rising to sponge_tau."""
import numpy as np
import pytest

from golden_io import load_reach_case, load_step_case
from parity_util import case_arrays
from test_gpu_parity import _require_gpu, errors, make_solver

pytestmark = pytest.mark.gpu

SPONGE = (24, 0.56)
TOL_U, TOL_RHO = 1e-5, 1e-5


def sponge_oracle(c, precision="f32"):
    from oracle.oracle import OracleLBM
    solid, F, cf, _ = case_arrays(c)
    o = OracleLBM(solid, *F, c.uin_lb, c.tau0, c.cs, cf, precision=precision, sponge=SPONGE)
    if "csmag2" in c.d:
        o.csmag2 = float(c.d["csmag2"])
    return o


@pytest.mark.parametrize("tile", ((3, 2, 4, 0, 0), (3, 4, 4, 0, 0)))
def test_sponge_float32_vs_oracle_config1(tile):
    """Config-1 lattice (192 x 50 x 12), wall model, full forcing, 24-column sponge: N = 1, 2, 5."""
    _require_gpu()
    c = load_reach_case("cfg1")
    L = make_solver(c, tile=tile, sponge=SPONGE)
    O = sponge_oracle(c)
    done = 0
    for n in (1, 2, 5):
        O.update_uref(c.bedwall)
        O.step(n - done)
        L.step(n - done)
        done = n
        eu, er = errors(L, O)
        assert eu < TOL_U and er < TOL_RHO, (tile, n, eu, er)
    assert L.status() == 0


@pytest.mark.parametrize("storage", ("fp32", "fp16"))
def test_sponge_changes_only_the_sponge_columns(storage):
    """Three steps with and without the sponge: identical fields left of the sponge (less the
    three columns three steps can carry a difference across), different inside it.  (From the
    equilibrium start the first collision has no non-equilibrium part, so the relaxation time
    shows from the second step on.)"""
    _require_gpu()
    c = load_step_case("mini_cfg1")
    a = make_solver(c, storage=storage)
    b = make_solver(c, storage=storage, sponge=(8, 0.7))
    a.step(3)
    b.step(3)
    for k in ("rho", "ux", "uy", "uz"):
        ga, gb = (getattr(L, k).cpu().numpy().reshape(L.nz, L.ny, L.nx) for L in (a, b))
        assert np.array_equal(ga[..., :a.nx - 8 - 3], gb[..., :a.nx - 8 - 3]), k
    ux_a, ux_b = (L.ux.cpu().numpy().reshape(L.nz, L.ny, L.nx)[..., -8:] for L in (a, b))
    assert not np.array_equal(ux_a, ux_b)


def test_sponge_float64_solver_vs_oracle():
    """fp64.Solver64 with the sponge against the float64 oracle with it, 40 steps of config 1."""
    _require_gpu()
    from test_accuracy_fp64 import _oracle_run
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.fp64 import Solver64
    import oracle.oracle as om
    reach = config1_case()
    orig = om.OracleLBM.__init__

    def with_sponge(self, *a, **k):
        k.setdefault("sponge", SPONGE)
        orig(self, *a, **k)
    om.OracleLBM.__init__ = with_sponge
    try:
        O = _oracle_run(reach, 40, "f64")
    finally:
        om.OracleLBM.__init__ = orig
    S = Solver64(reach, sponge=SPONGE)
    S.advance(40)
    r, u, v, w, _ = S.fields()
    umax = float(np.abs(O.ux).max())
    for got, want in ((u, O.ux), (v, O.uy), (w, O.uz)):
        assert np.abs(got - want).max() <= 1e-11 * umax
    assert np.abs(r - O.rho).max() <= 1e-12


def test_sponge_needs_the_split_pipeline():
    _require_gpu()
    from water_flow_simulation_b200 import _native as nat
    c = load_step_case("mini_cfg1")
    L = make_solver(c, tile=(0, 2, 4, 0, 0), sponge=(8, 0.7))
    with pytest.raises(nat.LBMError, match="split pipeline"):
        L.step(1)
