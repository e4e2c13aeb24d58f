"""Learned warm start end to end: seeded boat cases, LBM steady states, training, evaluation.

No counterpart in the reference (its runs always start from the 1D inlet profile and run a
fixed t_total of one flow-through, averaging the trailing 40%, floodsim/reach3d.py:398-467).

* `random_case(seed)` -- a seeded boat case from the ranges of the batched-ensemble
  benchmark: boat type (long-tail, outboard, tug, float pusher, high- and medium-pressure
  jets, water curtain), stage 2-4 m, bank slope 0-2, Manning n 0.025-0.035, one or two
  boats abreast or in line, propeller tilt 0-20 deg; at dx = 0.25 m on 40-64 m reaches.
* `generate(seeds)` -- runs the cases as a batch (16-bit storage) to their t_total with the
  reference's time averaging and returns (features, grid, target, mask) per case: the
  network learns the time-averaged flow the LBM itself produces.
* `train(net, data)` -- Adam over the cases, one case per step, in random order.
* `warm_start(run, net)` -- the network's prediction lifted to equilibrium populations and
  fields (lbm_lift_coarse) as the run's start state.
* `evaluate(net, seeds)` -- the reference protocol (plain float32 single-case runs to t_total)
  against the chosen method (warm start + 16-bit + batched, run to `frac` of t_total with the
  same trailing averaging) and against the same shortened run without the warm start:
  lid-level error (cm) of each against the reference protocol, and cases per hour.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import _native as nat
from .batch import CHUNK, BatchRun
from .geometry import Section, manning_discharge
from .reach3d import BOAT_TYPES, G, Fleet, ReachConfig, Run3D, build_reach, profiles_device
from .surrogate import FACTOR, N_OUT, RHO_SCALE, U_SCALE, SurrogateNet, case_features, case_targets

TYPES = ("longtail", "outboard", "tug", "pontoon", "jet_hp", "jet_mp", "curtain")


def _boat(key):
    return next(b for b in BOAT_TYPES if b.key == key) if isinstance(BOAT_TYPES, (list, tuple)) else BOAT_TYPES[key]


def random_case(seed, dx=0.25):
    """A seeded boat case (Reach) of the batched-ensemble ranges on a small lattice."""
    from dataclasses import replace
    rng = np.random.default_rng(seed)
    h = float(rng.uniform(2.0, 4.0))
    z = float(rng.choice([0.0, 1.0, 2.0]))
    B = float(rng.uniform(8.0, 16.0))
    n = float(rng.uniform(0.025, 0.035))
    S = 3e-4
    sec = Section(B=B, Hb=h, z=z, Bf=0.0, n=n)
    Q = manning_discharge(sec, h, S)
    boat = _boat(TYPES[int(rng.integers(len(TYPES)))])
    scale = min(1.0, 0.5 * h / max(boat.draft + boat.prop_depth, 0.5))          # fit the boat to the stage
    boat = replace(boat, tilt_deg=float(rng.uniform(0.0, 20.0)) if boat.prop_D > 0 else 0.0,
                   hull_L=min(boat.hull_L, 12.0), hull_B=min(boat.hull_B, 0.35 * B),
                   draft=boat.draft * scale, prop_depth=max(boat.prop_depth * scale, 0.3),
                   prop_D=min(boat.prop_D, 0.4 * h))
    count = int(rng.integers(1, 3))
    abreast = bool(rng.integers(2))
    length = float(rng.uniform(40.0, 64.0))
    fleet = Fleet(boat, rows=1 if abreast else count, per_row=count if abreast else 1,
                  row_spacing=boat.hull_L + 6.0, x_first=0.3 * length)
    cfg = ReachConfig(length=length, dx=dx, cs=0.17)
    return build_reach(sec, h, Q, S, fleet, cfg)


def _fields_mean(run):
    L = run.lbm
    n = max(L.navg, 1)
    return [L.avg_sum(k).cpu().numpy() / n for k in ("rho", "ux", "uy", "uz")]


def generate(seeds, batch_size=64, log=None):
    """[(features, dims, target, mask)] of the cases `seeds`, from batched LBM runs to t_total."""
    data = []
    for s0 in range(0, len(seeds), batch_size):
        reaches = [random_case(s) for s in seeds[s0:s0 + batch_size]]
        B = BatchRun(reaches)
        t0 = time.time()
        B.run_to_end()
        status = B.status()
        for r, run, st in zip(reaches, B.runs, status):
            if st:                       # a non-finite density: not a steady state to learn from
                continue
            uin = (r.uin_phys / r.vel).astype(np.float32)
            feat, dims = case_features(r.solid, r.Fx, r.Fy, r.Fz, uin, r.cf)
            target, mask = case_targets(r.solid, uin, *_fields_mean(run))
            data.append((feat, dims, target, mask))
        if log:
            log(f"generated {len(data)}/{len(seeds)} cases ({B.cells / 1e6:.1f}M cells, {time.time() - t0:.1f} s, "
                f"{sum(1 for x in status if x)} unstable dropped)")
    return data


def target_scale(data):
    """Per-channel RMS of the training targets over fluid voxels (the network predicts t / scale)."""
    num = sum((m[:, None] * t ** 2).sum(0) for _, _, t, m in data)
    den = sum(m.sum() for _, _, _, m in data)
    return np.sqrt(num / max(den, 1.0)).astype(np.float32) + np.float32(1e-6)


def train(net, data, epochs=20, lr=1e-3, seed=0, log=None):
    """Adam over the cases (one per step), cosine-decayed learning rate; returns per-epoch mean loss
    (in units of the per-channel target scale, which is stored in net.out_scale)."""
    torch = net.torch
    dev = net.device
    net.out_scale = target_scale(data)
    sc = net.out_scale[None, :]
    tensors = [(torch.as_tensor(f, device=dev), d, torch.as_tensor(t / sc, device=dev), torch.as_tensor(m, device=dev))
               for f, d, t, m in data]
    rng = np.random.default_rng(seed)
    total = epochs * len(tensors)
    it = 0
    history = []
    for ep in range(epochs):
        losses = []
        for k in rng.permutation(len(tensors)):
            f, d, t, m = tensors[k]
            net.zero_grad()
            loss, _ = net.loss_and_grad(f, d, t, m)
            net.adam(lr=lr * 0.5 * (1 + math.cos(math.pi * it / total)))
            losses.append(loss)
            it += 1
        net.check()
        history.append(float(torch.stack(losses).mean()))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.4f}")
    return history


def predict(net, reach):
    uin = (reach.uin_phys / reach.vel).astype(np.float32)
    feat, dims = case_features(reach.solid, reach.Fx, reach.Fy, reach.Fz, uin, reach.cf)
    out = net.forward(net.torch.as_tensor(feat, device=net.device), dims)
    return out, dims


def warm_start(run, net, density=True):
    """Replace the run's 1D-profile start by the network's prediction (populations and fields);
    density=False keeps rho = 1 and lifts the predicted velocity only."""
    import ctypes
    torch = net.torch
    L = run.lbm
    out, (Z, Y, X) = predict(net, run.r)
    out[:, :4] *= torch.as_tensor(net.out_scale, device=out.device)
    if not density:
        out[:, 3] = 0.0
    f = torch.empty(19 * L.cells, dtype=torch.float32, device=L.device)
    lat = L._lattice()
    nat.check(L.lib.lbm_lift_coarse(ctypes.byref(lat), out.data_ptr(), N_OUT, X, Y, Z, FACTOR, U_SCALE, RHO_SCALE,
                                    f.data_ptr(), L._stream()), "lbm_lift_coarse")
    L.load_populations(f)
    L._colU.zero_()


def _level_profile(run):
    return profiles_device(run, mean=True)["eta"]


def _eta_cm(reach, level):
    """Lid level (rho - 1 per x, lattice units) -> water level referenced to the outlet, cm."""
    eta = level / 3.0 * reach.vel ** 2 / G
    return 100.0 * (eta - eta[-1])


def evaluate(net, seeds, tol=5e-3, check_every=100, window=40, max_flows=3.0, level_tol_cm=0.5, ref_flows=2.0,
             density=True, ramp=False, log=None):
    """Held-out cases: the reference protocol against the chosen method, and the chosen method
    against the same batched run without the network.

    reference  float32, one case at a time, to t_total (one flow-through) with the trailing
               40% time average (floodsim/reach3d.py:398-467); the level answer eta_ref(x)
               is the same protocol run for `ref_flows` flow-throughs, and the one-flow-through
               result's own difference from it is reported as the protocol's noise floor;
    warm       the network's start state, 16-bit storage, all cases in one batch, each run
               until its discharge sum, sampled every `check_every` steps, changes by less
               than `tol` between the means of its last two windows of `window` samples and
               the window-mean lid level by less than `level_tol_cm`; the level answer is the
               mean over the last window.  A case that has not converged
               after `max_flows` flow-throughs is run again from the 1D start (fallback);
    cold       the same batched convergence run from the 1D start.
    ramp: the warm start keeps the cold start's force ramp (the boat forcing rises from zero
    over t_ramp, floodsim/reach3d.py:424-453) instead of applying the full forcing at once.
    Returns per-case steps to convergence, level errors (cm, max over x against eta_ref),
    wall times and cases per hour."""
    torch = net.torch
    reaches = [random_case(s) for s in seeds]
    t0 = time.time()
    one_eta, kept, ref_steps = [], [], 0
    for r in reaches:
        run = Run3D(r)
        n = int(math.ceil(run.t_total / r.dt / CHUNK)) * CHUNK
        run.advance(n)
        ref_steps += n
        if run.lbm.status() == 0:
            kept.append(r)
            one_eta.append(100.0 * _level_profile(run))
    torch.cuda.synchronize()
    t_ref = time.time() - t0
    dropped = len(reaches) - len(kept)
    reaches = kept
    ref_eta = []                        # the level answer: the protocol over ref_flows flow-throughs
    for r in reaches:
        run = Run3D(r)
        run.t_total *= ref_flows
        run.t_avg = run.t_total * (1 - r.cfg.avg_frac)
        run.advance(int(math.ceil(run.t_total / r.dt / CHUNK)) * CHUNK)
        ref_eta.append(100.0 * _level_profile(run))
    noise = [float(np.abs(a - b).max()) for a, b in zip(one_eta, ref_eta)]

    def converge(use_net, cases):
        B = BatchRun(cases, tol=tol, check_every=check_every, window=window, level_tol_cm=level_tol_cm)
        for i, run in enumerate(B.runs):
            B.target[i] = int(math.ceil(max_flows * run.t_total / run.r.dt / CHUNK)) * CHUNK
            if use_net:
                warm_start(run, net, density=density)
                if not ramp:             # the predicted flow already carries the full boat forcing
                    run._ramp_done = True
                    run.lbm.force_scale = 1.0
        B._rebatch()
        torch.cuda.synchronize()
        t1 = time.time()
        B.run_to_end()
        return B, time.time() - t1

    Bw, t_warm = converge(True, reaches)
    fallback = [i for i in range(len(reaches)) if not Bw.converged[i]]
    t_fb = 0.0
    warm_level = [_eta_cm(r, Bw.window_level(i)) for i, r in enumerate(reaches)]
    warm_steps = list(Bw.steps_done)
    if fallback:
        Bf, t_fb = converge(False, [reaches[i] for i in fallback])
        for k, i in enumerate(fallback):
            warm_level[i] = _eta_cm(reaches[i], Bf.window_level(k))
            warm_steps[i] += Bf.steps_done[k]
    Bc, t_cold = converge(False, reaches)
    cold_level = [_eta_cm(r, Bc.window_level(i)) for i, r in enumerate(reaches)]
    err = lambda lv: [float(np.abs(a - b).max()) for a, b in zip(lv, ref_eta)]  # noqa: E731
    res = dict(cases=len(reaches), unstable_dropped=dropped, tol=tol, window_steps=window * check_every, ramp=ramp,
               level_tol_cm=level_tol_cm, ref_flows=ref_flows, protocol_noise_cm=noise,
               ref_seconds=t_ref, ref_steps=ref_steps,
               warm_seconds=t_warm + t_fb, warm_steps=warm_steps, warm_converged=list(Bw.converged),
               fallback_cases=len(fallback),
               cold_seconds=t_cold, cold_steps=list(Bc.steps_done), cold_converged=list(Bc.converged),
               level_err_cm_warm=err(warm_level), level_err_cm_cold=err(cold_level),
               cases_per_hour_ref=3600 * len(reaches) / t_ref,
               cases_per_hour_warm=3600 * len(reaches) / (t_warm + t_fb),
               cases_per_hour_cold=3600 * len(reaches) / t_cold)
    if log:
        log(f"reference {t_ref:.1f} s ({ref_steps} steps); warm {t_warm + t_fb:.1f} s ({sum(warm_steps)} steps, "
            f"{len(fallback)} fallbacks); cold {t_cold:.1f} s ({sum(Bc.steps_done)} steps); level error max: warm "
            f"{max(res['level_err_cm_warm']):.2f} cm, cold {max(res['level_err_cm_cold']):.2f} cm, one-flow-through "
            f"protocol {max(noise):.2f} cm")
    return res
