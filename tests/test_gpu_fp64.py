"""The float64 GPU solver (lbm_step_f64 / lbm_bc_f64 / lbm_update_uref_f64, fp64.Solver64)
against the CPU float64 oracle (needs a B200).

Solver64 is the float64 reference of the accuracy statements at sizes the CPU oracle cannot
run; it must be the oracle's algorithm: the same fields after Run3D-cadence chunks (force
ramp, column-mean wall speed) to float64 rounding.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _require_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")


@pytest.mark.parametrize("steps", (1, 40))
def test_fp64_solver_matches_cpu_fp64_oracle(steps):
    """config-1 boat case (192 x 50 x 12, wall model, actuator disk): after 1 step and after
    two 20-step chunks, every field within 1e-11 of max|u| (velocity) / 1e-12 (density and
    populations)."""
    _require_gpu()
    from test_accuracy_fp64 import _oracle_run
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.fp64 import Solver64
    reach = config1_case()
    O = _oracle_run(reach, steps, "f64")
    S = Solver64(reach)
    S.advance(steps)
    r, u, v, w, _ = S.fields()
    umax = float(np.abs(O.ux).max())
    for got, want in ((u, O.ux), (v, O.uy), (w, O.uz)):
        assert np.abs(got - want).max() <= 1e-11 * umax
    assert np.abs(r - O.rho).max() <= 1e-12
    assert np.abs(S.f.cpu().numpy() - O.f).max() <= 1e-12


def test_fp64_solver_closed_box_stays_at_rest():
    """No inflow, no force, no wall model: a closed box at rest stays at rest to float64
    rounding."""
    _require_gpu()
    import torch
    from water_flow_simulation_b200 import _native as nat
    nz, ny, nx = 6, 7, 9
    N = nx * ny * nz
    dev = torch.device("cuda")
    lib = nat.load()
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
    rest = torch.tensor(np.repeat(w, N), dtype=torch.float64, device=dev)
    f, f2 = rest.clone(), torch.zeros_like(rest)
    z = lambda: torch.zeros(N, dtype=torch.float64, device=dev)  # noqa: E731
    solid = torch.zeros(N, dtype=torch.uint8, device=dev)
    Fx, Fy, Fz, rho, ux, uy, uz, cfw, uref = (z() for _ in range(9))
    p = lambda a: a.data_ptr()  # noqa: E731
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(10):
        assert lib.lbm_step_f64(p(f), p(f2), p(solid), p(Fx), p(Fy), p(Fz), p(rho), p(ux), p(uy), p(uz), p(cfw),
                                p(uref), nx, ny, nz, 0.6, 0.0289, 0, 0.0, st) == 0
        f, f2 = f2, f
    torch.cuda.synchronize()
    assert float((f - rest).abs().max()) <= 1e-15
    assert float((rho - 1).abs().max()) <= 1e-14
    assert float(ux.abs().max()) <= 1e-15
