"""Water-level and bed-shear error of the float32 and 16-bit paths against a float64 run.

The readouts are the reference's (floodsim/reach3d.py:192-193, 545-568, 571-618): the lid
water level eta(x) = (rho - 1)/3 (dx/dt)^2 / g averaged over the top layer's fluid cells and
referenced to the outlet, and the bed shear tau = rho_w cf |u|^2 of the first fluid cell
above the bed with cf from the Manning roughness height.  Compared, per case:

* level_max_cm: the largest |eta - eta_64| along the reach;
* drop_cm: the difference of the upstream level drop eta(x_up) - eta(outlet) that `compare`
  reports (x_up at 8 % of the length);
* shear_max_rel: the difference of the largest bed shear, relative to it;
* shear_mean_rel: the mean |tau - tau_64| over the bed, relative to the mean shear.

The float64 run is `fp64.Solver64` (GPU); at config-1 sizes the tests also check it against
the CPU float64 oracle.  Command line:

    python -m water_flow_simulation_b200.accuracy --workload reach36m --steps 20000
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def level_and_shear(reach, rho, ux, uy, uz, sp=None):
    """eta(x) in m (referenced to the outlet) and the bed shear map max over z (Pa), from
    host fields in the reference layout; `sp` is the speed field when it is a time average
    rather than |u| of the given velocity."""
    from .reach3d import G, RHO, log_cf, manning_ks
    sh = reach.solid.shape
    rho, ux, uy, uz = (np.asarray(a, np.float64).reshape(sh) for a in (rho, ux, uy, uz))
    fl = ~reach.solid
    top = fl[-1]
    eta = (rho[-1] - 1.0) / 3.0 * reach.vel ** 2 / G
    eta_x = (eta * top).sum(0) / np.maximum(top.sum(0), 1)
    if sp is None:
        sp2 = (ux * ux + uy * uy + uz * uz) * reach.vel ** 2
    else:
        sp2 = np.asarray(sp, np.float64).reshape(sh) ** 2 * reach.vel ** 2
    below = np.concatenate([np.ones((1,) + fl.shape[1:], bool), ~fl[:-1]], 0)
    first = fl & below
    tau = np.where(first, RHO * log_cf(0.5 * reach.dx, manning_ks(reach.sec.n)) * sp2, 0.0).max(axis=0)
    return eta_x - eta_x[-1], tau


def errors(eta, tau, eta_ref, tau_ref):
    """level_max_cm: largest |eta - eta_ref| along the reach; drop_cm: difference of the upstream
    level drop; shear_max_rel: of the largest bed shear; shear_avg_rel: of the bed-averaged shear
    (the mean of the bed-shear map); shear_mean_rel: the pointwise mean |tau - tau_ref| over the
    bed, relative to the mean shear."""
    i_up = max(int(0.08 * len(eta)), 1)
    bed = tau_ref > 0
    return dict(level_max_cm=100 * float(np.abs(eta - eta_ref).max()),
                drop_cm=100 * float(abs((eta[i_up] - eta[-1]) - (eta_ref[i_up] - eta_ref[-1]))),
                shear_max_rel=float(abs(tau.max() - tau_ref.max()) / tau_ref.max()),
                shear_avg_rel=float(abs(tau[bed].mean() - tau_ref[bed].mean()) / tau_ref[bed].mean()),
                shear_mean_rel=float(np.abs(tau - tau_ref)[bed].mean() / tau_ref[bed].mean()))


def _perturb(run, rel=1e-7, seed=1):
    """Multiply the start populations by 1 + rel * N(0, 1) (float32 storage): a second
    trajectory of the same case, for the spread a chaotic flow's readouts have by themselves."""
    import torch
    g = torch.Generator(device=run.lbm.f.device).manual_seed(seed)
    noise = torch.randn(run.lbm.f.shape, generator=g, device=run.lbm.f.device, dtype=torch.float32)
    run.lbm.f.mul_(1 + rel * noise)
    run.lbm.f2.copy_(run.lbm.f)


def against_fp64(reach, steps, storages=("fp32", "fp16"), average=False, log=None, save=None, sponge=None,
                 reference="fp64", avg_from=None):
    """Run the case `steps` steps in float64 and with each storage; returns {storage: errors}
    plus the wall seconds of each run.  With `average`, compares the time averages of the
    trailing window (the case must reach t_avg within `steps`; `avg_from`: the step the
    averaging starts at instead of the case's own t_avg).  A storage "fp32p" is float32 from a
    perturbed start (`_perturb`), "fp64p" float64 from a start perturbed by half a float32 ulp
    (`Solver64.perturb`): the spread of the readouts themselves.  `save`: an .npz path for every run's eta(x), bed
    shear map and, when averaged, its profiles (for the boat effects between a boat run and its base run,
    `level_change`)."""
    import torch
    from .fp64 import Solver64
    from .reach3d import Run3D, profiles_device, profiles_from_sums
    keys = ("rho", "ux", "uy", "uz", "sp", "uxx")

    def fp64_profiles(S):                  # the float64 run's time averages through profiles()
        return profiles_from_sums(reach, {k: a.cpu().numpy() for k, a in zip(keys, S.sums)}, S.navg)

    profs = {}
    out = {"steps": steps, "cells": int(reach.solid.size), "average": bool(average), "seconds": {},
           "avg_from": avg_from}
    t_avg = None if avg_from is None else (avg_from - 0.5) * reach.dt
    saved = {}
    t0 = time.time()
    if reference == "fp32":                       # a float32 run as the reference (no float64 run)
        run = Run3D(reach, storage="fp32", sponge=sponge)
        if t_avg is not None:
            run.t_avg = t_avg
        run.advance(steps)
        p = profiles_device(run, mean=average)
        ref, navg = (p["eta"], p["tau_bed"]), run.navg
        del run
    else:
        S = Solver64(reach, sponge=sponge)
        S.advance(steps, average=average, t_avg=t_avg)
        r, u, v, w, sp = S.fields(mean=average)
        navg = S.navg
        if average:
            profs[reference] = fp64_profiles(S)
        del S
        ref = level_and_shear(reach, r, u, v, w, sp=sp if average else None)
        del r, u, v, w, sp
    torch.cuda.synchronize()
    out["seconds"][reference] = time.time() - t0
    out["reference"] = reference
    torch.cuda.empty_cache()
    saved[reference + "_eta"], saved[reference + "_tau"] = ref
    if log:
        log(f"{reference}: {out['seconds'][reference]:.1f} s")
    for storage in storages:
        t0 = time.time()
        if storage == "fp64p":
            S = Solver64(reach, sponge=sponge)
            S.perturb()
            S.advance(steps, average=average, t_avg=t_avg)
            r, u, v, w, sp = S.fields(mean=average)
            eta, tau = level_and_shear(reach, r, u, v, w, sp=sp if average else None)
            n_out, status = S.navg, 0
            if average:
                profs[storage] = fp64_profiles(S)
            del S, r, u, v, w, sp
        else:
            run = Run3D(reach, storage="fp32" if storage == "fp32p" else storage, sponge=sponge)
            if storage == "fp32p":
                _perturb(run)
            if t_avg is not None:
                run.t_avg = t_avg
            run.advance(steps)
            p = profiles_device(run, mean=average)
            eta, tau = p["eta"], p["tau_bed"]
            if average:
                profs[storage] = p
            n_out, status = run.navg, int(run.lbm.status())
            del run
        torch.cuda.synchronize()
        out["seconds"][storage] = time.time() - t0
        if average and n_out != navg:
            raise RuntimeError(f"averaged outputs differ: {n_out} vs {navg}")
        out[storage] = errors(eta, tau, *ref)
        out[storage]["status"] = status
        saved[storage + "_eta"], saved[storage + "_tau"] = eta, tau
        if log:
            log(f"{storage}: {out[storage]}")
        torch.cuda.empty_cache()
    out["navg"] = navg
    if save:
        for k, p in profs.items():
            saved.update({f"{k}_prof_{name}": np.asarray(p[name]) for name in PROFILE_SAVE})
        np.savez_compressed(save, x=reach.x, **saved)
    return out


PROFILE_SAVE = ("x", "eta", "us", "umax", "q", "tau_bed", "mom")
# compare() outputs whose error against float64 the accuracy statement states
EFFECT_KEYS = ("d_eta_cm", "dQ_net_pct", "F_net_kN", "us_gain_pct", "tau_max", "umax")


def boat_effects(boat_npz, base_npz, reach):
    """compare() (floodsim/reach3d.py:571-618) of every saved averaged run against its base run
    -- level change, discharge gain from the momentum-flux balance, net force, surface-speed gain,
    largest shear and speed -- and each quantity's difference from float64's (relative for
    the non-level ones)."""
    from .reach3d import compare
    a, b = np.load(boat_npz), np.load(base_npz)
    runs = sorted({k.split("_prof_")[0] for k in a.files if "_prof_" in k})
    res = {}
    for k in runs:
        pb = {n: a[f"{k}_prof_{n}"] for n in PROFILE_SAVE}
        pa = {n: b[f"{k}_prof_{n}"] for n in PROFILE_SAVE}
        c = compare(pb, pa, reach, reach.cfg)
        res[k] = {n: float(c[n]) for n in EFFECT_KEYS}
    ref = res.get("fp64")
    if ref:
        for k, v in res.items():
            v["error"] = {n: (v[n] - ref[n]) if n in ("d_eta_cm", "dQ_net_pct", "us_gain_pct")
                          else (v[n] - ref[n]) / max(abs(ref[n]), 1e-30) for n in EFFECT_KEYS}
    return res


def level_change(boat_npz, base_npz, reach):
    """The boat's level change d_eta as `compare` reports it (floodsim/reach3d.py:571-590:
    upstream-to-outlet level drop of the boat run minus that of the base run, upstream read
    at 8 % of the length or 10 m ahead of the first hull) for every saved run, and each
    run's difference from float64, in cm."""
    a, b = np.load(boat_npz), np.load(base_npz)
    x = a["x"]
    i_up = max(int(0.08 * len(x)), 1)
    if reach.hulls:
        i_up = max(min(i_up, int(np.searchsorted(x, min(hb[0] for hb in reach.hulls) - 10.0))), 1)
    runs = sorted({k[:-4] for k in a.files if k.endswith("_eta") and "_prof_" not in k})
    d = {k: 100 * float((a[k + "_eta"][i_up] - a[k + "_eta"][-1]) - (b[k + "_eta"][i_up] - b[k + "_eta"][-1]))
         for k in runs}
    return {k: dict(d_eta_cm=d[k], error_cm=d[k] - d["fp64"]) for k in runs}


def statement(steps, avg_from, storages=("fp64p", "fp32", "fp16"), log=None):
    """The accuracy statement of the benchmark case: reach36m with the tug and without it, each
    run `steps` steps in float64 and in every storage, time-averaged from step `avg_from`;
    per storage the boat run's errors against float64 and the error of the boat's level change
    d_eta (boat minus base, as `compare` reports it).  "fp64p" gives the floor."""
    import tempfile
    from .cases import config2_case
    out = {"workload": "reach36m (cases.config2_case) with and without the tug", "steps": steps,
           "avg_from": avg_from, "storages": list(storages)}
    paths = {}
    for tag, with_boat in (("boat", True), ("base", False)):
        reach = config2_case(with_boat=with_boat)
        paths[tag] = tempfile.mktemp(suffix=f"_{tag}.npz")
        out[tag] = against_fp64(reach, steps, storages=storages, average=True, save=paths[tag], avg_from=avg_from,
                                log=log)
        if tag == "boat":
            boat_reach = reach
    out["level_change"] = level_change(paths["boat"], paths["base"], boat_reach)
    out["boat_effects"] = boat_effects(paths["boat"], paths["base"], boat_reach)
    return out


def stability(seeds, storages=("fp32", "fp16"), sponge=None, every=2000, log=None):
    """Long-run stability of seeded ensemble cases (cases.ensemble_case): each case run alone to
    the step at which Run3D.run_to_end stops it, in each storage, with the status word read
    every `every` steps; returns per case and storage the steps run and the first step at which
    a non-finite or non-positive density was seen (None: stayed finite)."""
    import torch
    from .batch import run_to_end_steps
    from .cases import ensemble_case
    from .reach3d import Run3D
    out = []
    for seed in seeds:
        reach = ensemble_case(int(seed))
        target = run_to_end_steps(reach)
        row = {"seed": int(seed), "cells": int(reach.solid.size), "steps_to_t_total": target, "sponge": sponge}
        for storage in storages:
            run = Run3D(reach, storage=storage, sponge=sponge)
            bad = None
            while run.lbm.nstep < target:
                run.advance(min(every, target - run.lbm.nstep))
                if run.lbm.status() & 1:
                    bad = run.lbm.nstep
                    break
            row[storage] = {"steps": int(run.lbm.nstep), "first_nonfinite_by_step": bad}
            if log:
                log(f"case {seed} {storage}: {row[storage]}")
            del run
            torch.cuda.empty_cache()
        out.append(row)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", choices=("config1", "reach7m", "reach36m", "reach36m_base"), default="reach36m")
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--average", action="store_true", help="compare time averages (needs steps past t_avg)")
    ap.add_argument("--perturbed", action="store_true", help="add a float32 run from a perturbed start")
    ap.add_argument("--floor", action="store_true",
                    help="add a float64 run from a start perturbed by half a float32 ulp (the readouts' own spread)")
    ap.add_argument("--save", default=None, help=".npz for the runs' eta(x) and bed shear")
    ap.add_argument("--sponge", default=None, help="cols,tau: the optional outlet sponge for every run")
    ap.add_argument("--reference", choices=("fp64", "fp32"), default="fp64",
                    help="the run the others are compared with (fp32: no float64 run, 16-bit only)")
    ap.add_argument("--avg-from", type=int, default=None, help="step the time averaging starts at")
    ap.add_argument("--stability", default=None,
                    help="comma-separated ensemble seeds: run each to t_total in float32 and 16-bit and report "
                         "where a non-finite density first appears (with --sponge, with the outlet sponge)")
    ap.add_argument("--statement", default=None,
                    help="write the benchmark case's accuracy statement (boat and base runs, float64 floor, "
                         "level change) to this JSON path, with --steps and --avg-from")
    args = ap.parse_args(argv)
    if args.stability:
        sp = None if not args.sponge else (int(args.sponge.split(",")[0]), float(args.sponge.split(",")[1]))
        res = stability([int(v) for v in args.stability.split(",")], sponge=sp, log=lambda m: print(m, flush=True))
        print(json.dumps(res), flush=True)
        return 0
    if args.statement:
        res = statement(args.steps, args.avg_from if args.avg_from is not None else args.steps // 2,
                        log=lambda m: print(m, flush=True))
        with open(args.statement, "w") as fh:
            json.dump(res, fh, indent=1)
        print(json.dumps(res), flush=True)
        return 0
    from .cases import config1_case, config2_case
    reach = {"config1": config1_case, "reach7m": lambda: config2_case(length=30.0),
             "reach36m": config2_case, "reach36m_base": lambda: config2_case(with_boat=False)}[args.workload]()
    sponge = None if not args.sponge else (int(args.sponge.split(",")[0]), float(args.sponge.split(",")[1]))
    storages = ("fp32", "fp16", "fp32p") if args.perturbed else ("fp32", "fp16")
    if args.floor:
        storages = ("fp64p",) + storages
    if args.reference == "fp32":
        storages = ("fp16",)
    res = against_fp64(reach, args.steps, storages=storages, average=args.average, save=args.save, sponge=sponge,
                       reference=args.reference, avg_from=args.avg_from)
    res["sponge"] = sponge
    res["workload"] = args.workload
    res["lattice"] = [reach.nx, reach.ny, reach.nz]
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
