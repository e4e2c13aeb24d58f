"""Batched 16-bit solves (lbm_batch_step_h, BatchRun) against single-case runs (needs a B200).

The batch kernels run the single-case kernels' per-segment code on concatenated work lists,
so every case of a batch must come out bit for bit as the same case run alone with the same
tile -- one launch per kernel class per step or the whole chunk in one persistent cooperative
launch, with and without the chunk captured as a CUDA graph, and after the batch has been
rebuilt because another case left it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TILE = (3, 2, 4, 0, 0)


def _require_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _reaches():
    """Three uneven boat cases: the config-1 channel, a shorter narrower one, a wider trapezoid."""
    from water_flow_simulation_b200.cases import config1_case
    from water_flow_simulation_b200.geometry import Section
    from water_flow_simulation_b200.reach3d import BoatType, Fleet, ReachConfig, boat_type, build_reach
    boat = BoatType("custom", "long-tail style", hull_L=6.0, hull_B=1.6, draft=0.6, n_props=1, prop_D=0.30,
                    prop_depth=0.35, tilt_deg=8, prop_x=1.5, prop_spacing=0, power_kW=40)
    r2 = build_reach(Section(B=8, Hb=2.5, z=0, Bf=0, n=0.03), 2.5, 0.7 * 20, 3e-4,
                     Fleet(boat, rows=1, per_row=1, x_first=8.0), ReachConfig(length=33, dx=0.25, cs=0.12))
    r3 = build_reach(Section(B=10, Hb=3, z=2, Bf=0, n=0.025), 3.0, 30.0, 3e-4,
                     Fleet(boat_type("outboard"), rows=1, per_row=1, x_first=12.0),
                     ReachConfig(length=40, dx=0.25, cs=0.17))
    return [config1_case(), r2, r3]


def _single(reach, steps):
    from water_flow_simulation_b200.reach3d import Run3D
    run = Run3D(reach, tile=TILE, storage="fp16")
    run.advance(steps)
    return run


@pytest.mark.parametrize("graphs,persistent", ((False, False), (True, False), (False, True), (True, True)))
def test_batch_equals_single_cases(graphs, persistent):
    torch = _require_gpu()
    from water_flow_simulation_b200.batch import BatchRun
    reaches = _reaches()
    steps = 100
    B = BatchRun(reaches, tile=TILE, use_graphs=graphs, max_steps=steps, persistent=persistent)
    assert B.advance(steps) is False                       # every case reached its step target
    for i, r in enumerate(reaches):
        ref = _single(r, steps)
        got = B.runs[i]
        assert torch.equal(got.lbm.f.view(torch.int16), ref.lbm.f.view(torch.int16)), i
        for k in ("rho", "ux", "uy", "uz"):
            assert torch.equal(getattr(got.lbm, k), getattr(ref.lbm, k)), (i, k)
        assert got.lbm.status() == 0


def test_batch_with_outlet_sponge_equals_single_cases():
    """The optional outlet sponge in a batch: every case as the same case alone with it."""
    torch = _require_gpu()
    from water_flow_simulation_b200.batch import BatchRun
    from water_flow_simulation_b200.reach3d import Run3D
    reaches = _reaches()
    sponge, steps = (8, 0.6), 60
    B = BatchRun(reaches, tile=TILE, use_graphs=True, max_steps=steps, sponge=sponge)
    B.advance(steps)
    for i, r in enumerate(reaches):
        ref = Run3D(r, tile=TILE, storage="fp16", sponge=sponge)
        ref.advance(steps)
        assert torch.equal(B.runs[i].lbm.f.view(torch.int16), ref.lbm.f.view(torch.int16)), i
        plain = _single(r, steps)                           # and the sponge did act
        assert not torch.equal(plain.lbm.f.view(torch.int16), ref.lbm.f.view(torch.int16)), i


def test_rebatch_after_a_case_leaves():
    """Case 1 stops after 40 steps; the others continue in a rebuilt batch and still match."""
    torch = _require_gpu()
    from water_flow_simulation_b200.batch import BatchRun
    reaches = _reaches()
    B = BatchRun(reaches, tile=TILE, use_graphs=True, max_steps=80)
    B.target[1] = 40
    B.advance(80)
    assert B.steps_done == [80, 40, 80]
    for i, n in enumerate((80, 40, 80)):
        ref = _single(reaches[i], n)
        assert torch.equal(B.runs[i].lbm.f.view(torch.int16), ref.lbm.f.view(torch.int16)), i


def test_convergence_stop():
    """A case stops once its discharge sum changes by less than tol over check_every steps."""
    _require_gpu()
    from water_flow_simulation_b200.batch import BatchRun
    B = BatchRun(_reaches()[:2], tile=TILE, tol=1e9, check_every=20, max_steps=400)
    B.advance(400)
    assert B.converged == [True, True] and B.steps_to_converge == [40, 40]
    B2 = BatchRun(_reaches()[:1], tile=TILE, tol=0.0, check_every=20, max_steps=60)
    B2.advance(60)
    assert B2.converged == [False] and B2.steps_done == [60]


def test_batch_argument_errors():
    _require_gpu()
    import ctypes
    from water_flow_simulation_b200 import _native as nat
    lib = nat.load()
    b = nat.Batch()
    assert lib.lbm_batch_step_h(ctypes.byref(b), 0, 0, None, None) == -1
    assert b"lattices" in lib.lbm_last_error()
    b.count = 300
    assert lib.lbm_batch_step_h(ctypes.byref(b), 0, 0, None, None) == -1
    with pytest.raises(ValueError):
        from water_flow_simulation_b200.batch import BatchRun
        BatchRun(_reaches()[:1], tile=(3, 4, 4, 0, 0))


def test_autotuner_picks_a_candidate_and_restores_state():
    torch = _require_gpu()
    from water_flow_simulation_b200 import autotune
    from water_flow_simulation_b200.batch import BatchRun
    from water_flow_simulation_b200.reach3d import Run3D
    reaches = _reaches()
    run = Run3D(reaches[0], tile=TILE, storage="fp16")
    run.advance(40)
    f_before = run.lbm.f.clone()
    best, times = autotune.tune_single(run.lbm, steps=4, warmup=2)
    assert best in times and len(times) >= 3 and torch.equal(run.lbm.f, f_before)
    assert tuple(run.lbm.tile_key()) == best
    B = BatchRun(reaches, tile=TILE, max_steps=100)
    f0 = [r.lbm.f.clone() for r in B.runs]
    best_b, times_b = autotune.tune_batch(B, steps=4, warmup=2)
    assert best_b in times_b and all(torch.equal(r.lbm.f, a) for r, a in zip(B.runs, f0))
    B.advance(40)                                  # runs with the tuned tile
    assert B.status() == [0, 0, 0]


@pytest.mark.parametrize("persistent", (False, True))
def test_batch_averages_and_ramp_equal_single_cases(persistent):
    """With the force ramp inside (0, 1) and the time averaging on after 40 steps, the batch's
    populations, fields and six average sums equal the cases run alone, bit for bit."""
    torch = _require_gpu()
    from water_flow_simulation_b200.batch import BatchRun
    from water_flow_simulation_b200.reach3d import Run3D
    reaches = _reaches()
    steps = 120
    B = BatchRun(reaches, tile=TILE, use_graphs=True, max_steps=steps, persistent=persistent)
    for run in B.runs:
        run.t_ramp, run.t_avg = 50 * run.r.dt, 39.5 * run.r.dt
    B.advance(steps)
    for i, r in enumerate(reaches):
        ref = Run3D(r, tile=TILE, storage="fp16")
        ref.t_ramp, ref.t_avg = 50 * r.dt, 39.5 * r.dt
        ref.advance(steps)
        got = B.runs[i]
        assert got.navg == ref.navg == 5
        assert torch.equal(got.lbm.f.view(torch.int16), ref.lbm.f.view(torch.int16)), i
        assert torch.equal(got.lbm._avg, ref.lbm._avg), i
        assert torch.equal(got.lbm._colU, ref.lbm._colU), i
        assert got.lbm.status() == 0


def test_persistent_chunk_argument_errors():
    """The chunk's modes are checked on the host: inner steps without OUTPUT, the last with it."""
    _require_gpu()
    import ctypes
    from water_flow_simulation_b200 import _native as nat
    from water_flow_simulation_b200.batch import BatchRun
    B = BatchRun(_reaches()[:1], tile=TILE, max_steps=20)
    lib = nat.load()
    ref = ctypes.byref(B._batch)
    assert lib.lbm_batch_chunk_h(ref, 0, 20, nat.STEP_OUTPUT, nat.STEP_OUTPUT, B._sync.data_ptr(), None) == -1
    assert lib.lbm_batch_chunk_h(ref, 0, 20, 0, 0, B._sync.data_ptr(), None) == -1
    assert lib.lbm_batch_chunk_h(ref, 0, 20, 0, nat.STEP_OUTPUT, None, None) == -1
    assert lib.lbm_batch_chunk_h(ref, 0, 0, 0, nat.STEP_OUTPUT, B._sync.data_ptr(), None) == -1


def test_persistent_chunk_long_run_bit_identical():
    """A longer run on a benchmark-ensemble case (seed 23, 2.7M cells, 4000 steps, averaging on
    for the last 2000): the persistent chunk and the per-step launches stay bit-identical, so
    no read of data written earlier in the launch goes stale."""
    torch = _require_gpu()
    from water_flow_simulation_b200.batch import BatchRun
    from water_flow_simulation_b200.cases import ensemble_case
    reaches = [ensemble_case(23), _reaches()[0]]
    out = []
    for persistent in (False, True):
        B = BatchRun(reaches, tile=TILE, use_graphs=True, max_steps=4000, persistent=persistent)
        for run in B.runs:
            run.t_avg = 1999.5 * run.r.dt
        B.advance(4000)
        out.append(B)
    a, b = out
    for ra, rb in zip(a.runs, b.runs):
        assert ra.navg == rb.navg == 101
        assert torch.equal(ra.lbm.f.view(torch.int16), rb.lbm.f.view(torch.int16))
        assert torch.equal(ra.lbm._avg, rb.lbm._avg) and torch.equal(ra.lbm._colU, rb.lbm._colU)
        assert ra.lbm.status() == 0 and rb.lbm.status() == 0
