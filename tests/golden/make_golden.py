"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run once, with the reference source tree given by the FLOODSIM_REF environment
variable or as the first argument (there is no default):

    FLOODSIM_REF=<path to the floodsim checkout> python tests/golden/make_golden.py

Nothing at test time runs this script or reads the reference; the tests read
only the .npz files it writes.

The reference's lbm3d.py does not compile under numba 0.65 as shipped:
``float(wl[k])`` on a numba boolean raises NumbaTypeError (floodsim/lbm3d.py:226-228).
The loader below reads lbm3d.py as text, rewrites those six calls to
``(1.0 if wl[k] else 0.0)`` and ``cache=True`` to ``cache=False`` (the source
tree is read-only), and executes the result as module ``floodsim.lbm3d`` before
importing reach3d.  No arithmetic changes.

Fixtures written:

* ``reach_<case>.npz`` -- build_reach outputs (floodsim/reach3d.py:201-297) and
  wall_cf (reach3d.py:315-343) for several sections/boats: the bit-exact
  KATs for the host reach builder and for the cell flag maps.
* ``export_<case>.npz`` -- the web viewer's case export (floodsim/web3d.py:35-86,
  export_case after profiles, reach3d.py:545-568) of a reference Run3D whose
  time-average sums are seeded random fields: the sums, the count, the
  profiles arrays the export reads, and the exported dictionary as JSON.
* ``particles_<case>.npz`` -- the reference's tracer particles (init_particles and three
  move_particles calls, reach3d.py:499-541) through a seeded random velocity field with
  non-finite and fast cells: positions after each call.  Restarted particles come from
  the reference's unseeded generator; the tests compare the others bit for bit.
* ``readouts_<case>.npz`` -- the reference's ``profiles`` (every key) of a boat run and
  of its no-boat base run whose time-average sums are seeded fields with a jet behind the
  propellers, and ``compare`` of the two (floodsim/reach3d.py:545-618).
* ``advance_<case>.npz`` -- the reference's ``Run3D.advance`` (reach3d.py:424-453) in
  3-step chunks with the force ramp and the time averaging both active: ramp time and
  averaging start moved to a few steps, fields, uref and averaging sums after every chunk.
* ``steps_<case>.npz`` -- the reference's Numba solver state after N steps
  (floodsim/lbm3d.py:390-412 driven through Run3D.advance, reach3d.py:424-453,
  so uref is refreshed every 20 steps), on small lattices: rho/ux/uy/uz after
  N in {1, 2, 5, 25} and the full population array after 1 step.
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np

REF = os.environ.get("FLOODSIM_REF") or (sys.argv[1] if len(sys.argv) > 1 else None)
OUT = os.path.dirname(os.path.abspath(__file__))


def load_reference():
    if "floodsim.reach3d" in sys.modules:
        return
    if not REF:
        raise SystemExit("give the reference source tree: FLOODSIM_REF=<path> or the first argument")
    sys.path.insert(0, REF)
    import floodsim  # noqa: F401

    path = os.path.join(REF, "floodsim", "lbm3d.py")
    src = open(path, encoding="utf-8").read()
    for k in range(1, 7):
        src = src.replace(f"float(wl[{k}])", f"(1.0 if wl[{k}] else 0.0)")
    src = src.replace("cache=True", "cache=False")
    mod = types.ModuleType("floodsim.lbm3d")
    mod.__file__ = path
    exec(compile(src, path, "exec"), mod.__dict__)
    sys.modules["floodsim.lbm3d"] = mod
    import floodsim.reach3d  # noqa: F401


# name -> (section kwargs, h, Q, S, boat key or custom tuple, boat overrides, fleet kwargs, cfg kwargs)
REACH_CASES = {
    # the 48 m x 12 m x 3 m rectangular channel with one 10 m long-tail-style boat
    "cfg1": dict(sec=dict(B=12, Hb=3, z=0, Bf=0, n=0.03), h=3.0, Q=0.8 * 36, S=3e-4,
                 boat=("custom", dict(name="c", hull_L=10.0, hull_B=2.0, draft=0.8, n_props=1, prop_D=0.30,
                                      prop_depth=0.35, tilt_deg=12, prop_x=2.5, prop_spacing=0, power_kW=75)),
                 fleet=dict(rows=1, per_row=1, x_first=11.0), cfg=dict(length=48, dx=0.25, cs=0.12)),
    # trapezoid with two tugs abreast: two props each, under the stern (prop_x < 0)
    "tug_trap": dict(sec=dict(B=14, Hb=3.5, z=2, Bf=0, n=0.025), h=3.0, Q=60.0, S=2e-4,
                     boat=("tug", {}), fleet=dict(rows=1, per_row=2, x_first=12.0),
                     cfg=dict(length=60, dx=0.5, cs=0.17)),
    # over-bank stage with floodplains, 100 bar jets spread over three yaws
    "jet_flood": dict(sec=dict(B=10, Hb=2.0, z=1.5, Bf=3.0, n=0.03), h=2.5, Q=40.0, S=3e-4,
                      boat=("jet_hp", dict(spread_deg=30)), fleet=dict(rows=1, per_row=2, x_first=8.0),
                      cfg=dict(length=40, dx=0.25, cs=0.17)),
    # two rows of curtains, plain no-slip walls (wall model off)
    "curtain_nowm": dict(sec=dict(B=16, Hb=3, z=1, Bf=0, n=0.03), h=2.0, Q=30.0, S=2e-4,
                         boat=("curtain", {}), fleet=dict(rows=2, per_row=1, row_spacing=14.0, x_first=6.0),
                         cfg=dict(length=48, dx=0.5, wall_model=False)),
    # a deep draft in shallow water (draft clamp and prop-lift notes), outboard, auto dx
    "shallow_outboard": dict(sec=dict(B=8, Hb=1.5, z=0.5, Bf=0, n=0.035), h=0.8, Q=4.0, S=5e-4,
                             boat=("outboard", dict(draft=0.75, prop_depth=0.7)),
                             fleet=dict(rows=1, per_row=1, x_first=5.0), cfg=dict(length=30, max_cells=60_000)),
    # no boats at all (the base run of every test)
    "base_rect": dict(sec=dict(B=12, Hb=3, z=0, Bf=0, n=0.03), h=3.0, Q=0.8 * 36, S=3e-4,
                      boat=("longtail", {}), fleet=dict(rows=1, per_row=3, enabled=False),
                      cfg=dict(length=48, dx=0.5, cs=0.12)),
}

# small lattices stepped by the reference solver
STEP_CASES = {
    "mini_cfg1": dict(REACH_CASES["cfg1"], cfg=dict(length=32, dx=0.5, cs=0.12)),
    "mini_tug": dict(REACH_CASES["tug_trap"], cfg=dict(length=40, dx=0.5, cs=0.17)),
    "mini_jet": dict(REACH_CASES["jet_flood"], cfg=dict(length=24, dx=0.5, cs=0.17)),
    "mini_nowm": dict(REACH_CASES["cfg1"], cfg=dict(length=32, dx=0.5, cs=0.12, wall_model=False)),
}
STEP_NS = (1, 2, 5, 25)

# cases whose viewer export is recorded (odd and even ny / nx, boats, jets, floodplains)
EXPORT_CASES = {
    "mini_cfg1": STEP_CASES["mini_cfg1"],
    "mini_tug": STEP_CASES["mini_tug"],
    "jet_flood": dict(REACH_CASES["jet_flood"], cfg=dict(length=12.25, dx=0.25, cs=0.17)),
}


def make_reach(spec):
    from floodsim.geometry import Section
    from floodsim.reach3d import BoatType, Fleet, ReachConfig, boat_type, build_reach
    from dataclasses import replace

    key, over = spec["boat"]
    if key == "custom":
        b = BoatType("custom", **over)
    else:
        b = replace(boat_type(key), **over)
    fleet = Fleet(b, **spec["fleet"])
    cfg = ReachConfig(**spec["cfg"])
    sec = Section(**spec["sec"])
    return build_reach(sec, spec["h"], spec["Q"], spec["S"], fleet, cfg), cfg


def sparse(a):
    flat = np.ascontiguousarray(a).ravel()
    idx = np.flatnonzero(flat).astype(np.int64)
    return idx, flat[idx]


def reach_arrays(r, cfg):
    nu_lb = max(1e-6 * r.dt / r.dx ** 2, 2e-4)      # Run3D.__init__, reach3d.py:383
    out = dict(
        dims=np.array([r.nx, r.ny, r.nz], np.int64),
        scalars=np.array([r.dx, r.dt, r.V, r.A, r.W, r.h, r.Q, r.S, 0.5 + 3 * nu_lb, cfg.cs], np.float64),
        solid=np.packbits(r.solid.ravel()),
        uin_phys=np.asarray(r.uin_phys, np.float64),
        uin_lb=(r.uin_phys / r.vel).astype(np.float32),
        y=np.asarray(r.y, np.float64), zc=np.asarray(r.zc, np.float64),
    )
    for nm in ("Fx", "Fy", "Fz"):
        out[nm + "_idx"], out[nm + "_val"] = sparse(getattr(r, nm))
    if r.cf is not None:
        out["cf_idx"], out["cf_val"] = sparse(r.cf)
        out["bedwall"] = np.packbits(r.bedwall.ravel())
    meta = dict(hulls=[list(map(float, h)) for h in r.hulls],
                props={i: {k: float(v) for k, v in p.items()} for i, p in enumerate(r.props)},
                notes=r.notes, wall_model=bool(cfg.wall_model))
    out["meta"] = np.array(json.dumps(meta, ensure_ascii=False))
    return out


def run_steps(r, cfg):
    """Step the reference solver with full (unramped) forcing; uref refreshed
    before every 20-step chunk exactly as Run3D.advance does."""
    from floodsim.backend import Backend
    from floodsim.reach3d import Run3D

    # the numpy-backend LBM3D aliases the reach's force arrays and Run3D zeroes them for its ramp
    F0 = tuple(np.array(a, np.float32).ravel() for a in (r.Fx, r.Fy, r.Fz))
    run = Run3D(r, Backend())
    L = run.lbm
    L.Fx, L.Fy, L.Fz = F0
    run._ramp_done = True
    out = {}
    done = 0
    for n in STEP_NS:
        run.advance(n - done)
        done = n
        for nm in ("rho", "ux", "uy", "uz"):
            out[f"{nm}_{n}"] = np.array(getattr(L, nm), np.float32)
        if n == 1:
            out["f_1"] = np.array(L.f, np.float32)
    out["uref_25"] = np.array(L.uref, np.float32)
    out["tau0"] = np.array(L.tau0)
    out["csmag2"] = np.array(L.csmag2)
    return out


def export_arrays(r, seed):
    """Seed a reference Run3D's time-average sums, then run the reference's profiles and
    export_case on it."""
    from floodsim.backend import Backend
    from floodsim.reach3d import Run3D, profiles
    from floodsim.web3d import export_case

    run = Run3D(r, Backend())
    rng = np.random.default_rng(seed)
    navg = 37
    n = r.cells
    fl = ~r.solid.ravel()
    ux = (0.09 + 0.03 * rng.standard_normal(n)) * fl
    uy = 0.02 * rng.standard_normal(n) * fl
    uz = 0.01 * rng.standard_normal(n) * fl
    rho = np.where(fl, 1.0 + 2e-4 * rng.standard_normal(n), 1.0)
    sp = np.sqrt(ux * ux + uy * uy + uz * uz) + 0.004 * np.abs(rng.standard_normal(n)) * fl
    uxx = ux * ux + 1e-4 * np.abs(rng.standard_normal(n)) * fl
    for k, a in (("ux", ux), ("uy", uy), ("uz", uz), ("rho", rho), ("sp", sp), ("uxx", uxx)):
        run.sum[k] = (a * navg).astype(np.float32)
    run.navg = navg
    res = profiles(run)
    out = export_case(run, "case", None, res)
    arrays = {f"sum_{k}": v for k, v in run.sum.items()}
    arrays.update(navg=np.array(navg), res_x=res["x"], res_eta=res["eta"], res_umax=res["umax"],
                  res_tau_bed=res["tau_bed"], export=np.array(json.dumps(out)))
    return arrays


def particle_arrays(r, seed, n=600, dts=(0.05, 0.2, 0.5)):
    from floodsim.backend import Backend
    from floodsim.reach3d import Run3D

    run = Run3D(r, Backend())
    L = run.lbm
    rng = np.random.default_rng(seed)
    N = r.cells
    fl = ~r.solid.ravel()
    ux = ((0.05 + 0.03 * rng.standard_normal(N)) * fl).astype(np.float32)
    uy = (0.02 * rng.standard_normal(N) * fl).astype(np.float32)
    uz = (0.01 * rng.standard_normal(N) * fl).astype(np.float32)
    ux[rng.integers(0, N, 30)] = np.nan                     # non-finite velocities read as 0
    uy[rng.integers(0, N, 30)] = np.inf
    uz[rng.integers(0, N, 30)] = -np.inf
    ux[rng.integers(0, N, 200)] = 3.0                       # fast cells push particles out
    L.ux, L.uy, L.uz = ux, uy, uz
    run.init_particles(n)
    out = dict(ux=ux, uy=uy, uz=uz, dts=np.array(dts), P0=run.P.copy())
    for k, dt in enumerate(dts):
        run.move_particles(dt)
        out[f"P{k + 1}"] = run.P.copy()
    return out


def _seeded_sums(r, rng, navg, jet_from=None):
    """Time-average sums of plausible fields: a sheared inflow, noise, and (if jet_from is
    given) a fast stream behind x = jet_from in the middle third of the width."""
    n = r.cells
    fl = ~r.solid.ravel()
    z, y, x = np.meshgrid(np.arange(r.nz), np.arange(r.ny), np.arange(r.nx), indexing="ij")
    base = 0.06 + 0.03 * (z.ravel() + 0.5) / r.nz
    jet = 0.0
    if jet_from is not None:
        mid = (np.abs(y.ravel() - r.ny / 2) < r.ny / 6) & (x.ravel() > jet_from)
        jet = np.where(mid, 0.12 * np.exp(-(x.ravel() - jet_from) / max(r.nx / 3, 1)), 0.0)
    ux = (base + jet + 0.01 * rng.standard_normal(n)) * fl
    uy = 0.01 * rng.standard_normal(n) * fl
    uz = 0.005 * rng.standard_normal(n) * fl
    rho = np.where(fl, 1.0 + 3e-4 * (1 - x.ravel() / r.nx) + 2e-5 * rng.standard_normal(n), 1.0)
    sp = np.sqrt(ux * ux + uy * uy + uz * uz) + 0.002 * np.abs(rng.standard_normal(n)) * fl
    uxx = ux * ux + 5e-5 * np.abs(rng.standard_normal(n)) * fl
    return {k: (a * navg).astype(np.float32) for k, a in
            (("ux", ux), ("uy", uy), ("uz", uz), ("rho", rho), ("sp", sp), ("uxx", uxx))}


def readout_arrays(spec, seed):
    """The reference's profiles of a boat run and of its base run (seeded sums) and compare."""
    from dataclasses import replace
    from floodsim.backend import Backend
    from floodsim.reach3d import Run3D, compare, profiles

    r, cfg = make_reach(spec)
    base_spec = dict(spec, fleet=dict(spec["fleet"], enabled=False))
    rb, _ = make_reach(base_spec)
    rng = np.random.default_rng(seed)
    out = {}
    res = {}
    for tag, reach in (("boat", r), ("base", rb)):
        run = Run3D(reach, Backend())
        navg = 23 if tag == "boat" else 19
        jet_from = int(max(p["x"] for p in reach.props) / reach.dx) if reach.props else None
        run.sum = _seeded_sums(reach, rng, navg, jet_from)
        run.navg = navg
        res[tag] = profiles(run)
        for k, v in run.sum.items():
            out[f"{tag}_sum_{k}"] = v
        out[f"{tag}_navg"] = np.array(navg)
        for k, v in res[tag].items():
            out[f"{tag}_res_{k}"] = np.asarray(v)
    c = compare(res["boat"], res["base"], r, cfg)
    out["compare"] = np.array(json.dumps({k: (v if not isinstance(v, float) or np.isfinite(v) else None)
                                          for k, v in c.items()}))
    out["base_spec"] = np.array(json.dumps(base_spec))
    return r, cfg, out


ADVANCE_CHUNKS = (3, 3, 3, 3)


def advance_arrays(r, cfg, ramp_steps=7, avg_from_step=5):
    """The reference's Run3D.advance in 3-step chunks with its force ramp over `ramp_steps`
    steps and its time averaging from step `avg_from_step` on (both moved from their case
    values so that a few steps cover them)."""
    from floodsim.backend import Backend
    from floodsim.reach3d import Run3D

    run = Run3D(r, Backend())
    assert not run._ramp_done, "the case needs propellers for a ramp"
    run.t_ramp = ramp_steps * r.dt
    run.t_avg = avg_from_step * r.dt
    L = run.lbm
    out = dict(t_ramp=np.array(run.t_ramp), t_avg=np.array(run.t_avg), chunks=np.array(ADVANCE_CHUNKS))
    for k, m in enumerate(ADVANCE_CHUNKS):
        run.advance(m)
        for nm in ("rho", "ux", "uy", "uz", "uref"):
            out[f"{nm}_c{k}"] = np.array(getattr(L, nm), np.float32)
        out[f"fx_scale_c{k}"] = np.array(float(np.float32(np.abs(L.Fx).max() / max(np.abs(run._F0[0]).max(), 1e-30))))
        out[f"navg_c{k}"] = np.array(run.navg)
        for nm, v in run.sum.items():
            out[f"sum_{nm}_c{k}"] = np.array(v, np.float32)
    return out


def main():
    load_reference()
    for k, name in enumerate(("mini_tug", "mini_cfg1")):
        spec = STEP_CASES[name]
        r, cfg, arrays = readout_arrays(spec, 300 + k)
        arrays.update(reach_arrays(r, cfg))
        np.savez_compressed(os.path.join(OUT, f"readouts_{name}.npz"), spec=np.array(json.dumps(spec)), **arrays)
        print("readouts", name, r.nx, r.ny, r.nz)
    for name in ("mini_tug", "mini_cfg1"):
        r, cfg = make_reach(STEP_CASES[name])
        arrays = reach_arrays(r, cfg)
        arrays.update(advance_arrays(r, cfg))
        np.savez_compressed(os.path.join(OUT, f"advance_{name}.npz"), spec=np.array(json.dumps(STEP_CASES[name])),
                            **arrays)
        print("advance", name, r.nx, r.ny, r.nz)
    if os.environ.get("GOLDEN_ONLY_NEW"):
        return
    for k, name in enumerate(("mini_cfg1", "mini_tug")):
        r, cfg = make_reach(STEP_CASES[name])
        arrays = reach_arrays(r, cfg)
        arrays.update(particle_arrays(r, 200 + k))
        np.savez_compressed(os.path.join(OUT, f"particles_{name}.npz"), spec=np.array(json.dumps(STEP_CASES[name])),
                            **arrays)
        print("particles", name, r.nx, r.ny, r.nz)
    for k, (name, spec) in enumerate(EXPORT_CASES.items()):
        r, cfg = make_reach(spec)
        arrays = reach_arrays(r, cfg)
        arrays.update(export_arrays(r, 100 + k))
        np.savez_compressed(os.path.join(OUT, f"export_{name}.npz"), spec=np.array(json.dumps(spec)), **arrays)
        print("export", name, r.nx, r.ny, r.nz)
    for name, spec in REACH_CASES.items():
        r, cfg = make_reach(spec)
        np.savez_compressed(os.path.join(OUT, f"reach_{name}.npz"), spec=np.array(json.dumps(spec)),
                            **reach_arrays(r, cfg))
        print("reach", name, r.nx, r.ny, r.nz, r.notes)
    for name, spec in STEP_CASES.items():
        r, cfg = make_reach(spec)
        arrays = reach_arrays(r, cfg)
        arrays.update(run_steps(r, cfg))
        np.savez_compressed(os.path.join(OUT, f"steps_{name}.npz"), spec=np.array(json.dumps(spec)), **arrays)
        print("steps", name, r.nx, r.ny, r.nz, r.nx * r.ny * r.nz)


if __name__ == "__main__":
    main()
