"""The recommended boat tests and their runner (floodsim/boat_tests.py), batched on the GPU.

`BOAT_TESTS` holds the reference's six tests -- boat type, boat count, water level,
propeller tilt, row layout, jets and curtains against propellers -- with the same variants
(boat, rows, boats per row, row spacing, level, parameter overrides) under short titles of
our own; the reference's descriptive prose is not carried.  `run_test` has the reference's signature and result list
(floodsim/boat_tests.py:73-113): every variant against the no-boat run at its water level,
`profiles` and `compare` of each, `on_result(c, run)` per variant in order.

What changes is how the runs are made.  The reference runs the base and boat cases one
after another in float32; here, by default, all of them -- one base per distinct level and
every boat variant -- advance together in one `BatchRun` with 16-bit populations (one
launch per kernel class per step, 20-step chunks replayed as CUDA graphs), each to the step
at which `Run3D.run_to_end` would stop it, and the profiles come from the float64 device
reductions.  `storage="fp32", batched=False` reproduces the reference's sequence exactly.
"""
from __future__ import annotations

from dataclasses import replace

from .reach3d import Fleet, ReachConfig, Run3D, boat_type, build_reach, compare, profiles, profiles_device

BOAT_TESTS = [
    dict(key="B1", title="B1 boat types",
         variants=[dict(label="long-tail x3", boat="longtail", rows=1, per_row=3),
                   dict(label="outboard x3", boat="outboard", rows=1, per_row=3),
                   dict(label="tug x3", boat="tug", rows=1, per_row=3),
                   dict(label="pusher pontoon x3", boat="pontoon", rows=1, per_row=3)]),
    dict(key="B2", title="B2 number of tugs",
         variants=[dict(label="tug x1", boat="tug", rows=1, per_row=1),
                   dict(label="tug x2", boat="tug", rows=1, per_row=2),
                   dict(label="tug x3", boat="tug", rows=1, per_row=3),
                   dict(label="tug 2 rows x3", boat="tug", rows=2, per_row=3, row_spacing=40)]),
    dict(key="B3", title="B3 stage",
         variants=[dict(label="low water", boat="longtail", rows=1, per_row=4, level="low"),
                   dict(label="middle water", boat="longtail", rows=1, per_row=4, level="mid"),
                   dict(label="high water", boat="longtail", rows=1, per_row=4, level="high")]),
    dict(key="B4", title="B4 shaft tilt",
         variants=[dict(label="tilt 0 deg", boat="longtail", rows=1, per_row=4, over=dict(tilt_deg=0)),
                   dict(label="tilt 12 deg", boat="longtail", rows=1, per_row=4, over=dict(tilt_deg=12)),
                   dict(label="tilt 25 deg", boat="longtail", rows=1, per_row=4, over=dict(tilt_deg=25))]),
    dict(key="B5", title="B5 rows",
         variants=[dict(label="1 row x 6", boat="longtail", rows=1, per_row=6),
                   dict(label="2 rows x 3", boat="longtail", rows=2, per_row=3, row_spacing=25),
                   dict(label="3 rows x 2", boat="longtail", rows=3, per_row=2, row_spacing=25)]),
    dict(key="B6", title="B6 jets and curtain vs propellers",
         variants=[dict(label="large propeller 100 kW x3", boat="pontoon", rows=1, per_row=3,
                        over=dict(power_kW=100)),
                   dict(label="100 bar jet, straight x3", boat="jet_hp", rows=1, per_row=3),
                   dict(label="100 bar jet, spread +-30 deg x3", boat="jet_hp", rows=1, per_row=3,
                        over=dict(spread_deg=30)),
                   dict(label="10 bar jet x3", boat="jet_mp", rows=1, per_row=3),
                   dict(label="3 m/s curtain x3", boat="curtain", rows=1, per_row=3)]),
]


def pick_level(levels, which, Hb):
    """floodsim/boat_tests.py:62-70: 'low' / 'high' = the lowest / highest level, 'mid' = the
    middle in-bank level; anything else is returned as it is."""
    lv = sorted(levels)
    inb = [h for h in lv if h <= Hb] or lv
    if which == "low":
        return lv[0]
    if which == "high":
        return lv[-1]
    return inb[len(inb) // 2] if which == "mid" else which


def _variant_reaches(test, sec, levels, h_sel, cfg, flow_fn, x_first, boat_edits):
    """(h, boat reach, fleet) per variant and the no-boat reach per distinct level, built
    as floodsim/boat_tests.py:81-101 builds them."""
    cases, bases = [], {}
    for v in test["variants"]:
        h = pick_level(levels, v["level"], sec.Hb) if "level" in v else h_sel
        Q, S = flow_fn(h)
        b = boat_type(v["boat"])
        if boat_edits and v["boat"] in boat_edits:
            b = replace(b, **boat_edits[v["boat"]])
        if "over" in v:
            b = replace(b, **v["over"])
        fleet = Fleet(b, rows=v["rows"], per_row=v["per_row"], row_spacing=v.get("row_spacing", 30.0),
                      x_first=x_first)
        if h not in bases:
            bases[h] = build_reach(sec, h, Q, S, replace(fleet, enabled=False), cfg)
        cases.append((h, build_reach(sec, h, Q, S, fleet, cfg), v))
    return cases, bases


def run_test(test, river, sec, levels, h_sel, cfg: ReachConfig, be, flow_fn, x_first=40.0,
             progress=None, cancel=None, on_result=None, boat_edits=None, *, storage="fp16", batched=True,
             tile=None, sponge=None):
    """Every variant of `test` against the no-boat run at the same level; returns the list of
    `compare` results with label, profiles, base_profiles and notes added (the reference's
    result list).  progress(fraction, label), cancel() and on_result(c, run) as in the
    reference; with `batched`, progress reports the whole batch and on_result is called after
    it, in variant order.  `sponge`: the optional outlet sponge (cols, tau) for every run."""
    if batched and storage != "fp16":
        raise ValueError("batched runs use 16-bit storage")
    cases, bases = _variant_reaches(test, sec, levels, h_sel, cfg, flow_fn, x_first, boat_edits)
    results = []
    n = len(cases)
    if not batched:                                 # the reference's sequence (floodsim/boat_tests.py:80-113)
        base_res = {}
        for k, (h, rr, v) in enumerate(cases):
            if cancel and cancel():
                break

            def prog(f, k=k, part=0, label=v["label"]):
                if progress:
                    progress((k + 0.5 * part + 0.5 * f) / n, label)

            read = profiles if storage == "fp32" else profiles_device
            if h not in base_res:
                run_b = Run3D(bases[h], be, tile=tile, storage=storage, sponge=sponge)
                run_b.run_to_end(progress=lambda f: prog(f, part=0), cancel=cancel)
                base_res[h] = read(run_b)
            run = Run3D(rr, be, tile=tile, storage=storage, sponge=sponge)
            run.run_to_end(progress=lambda f: prog(f, part=1), cancel=cancel)
            res = read(run)
            results.append(_result(res, base_res[h], rr, cfg, v))
            if on_result:
                on_result(results[-1], run)
        return results

    from .batch import BatchRun, run_to_end_steps
    levels_used = list(bases)
    reaches = [bases[h] for h in levels_used] + [rr for _, rr, _ in cases]
    B = BatchRun(reaches, tile=tile or (3, 2, 4, 0, 0), max_steps=[run_to_end_steps(r) for r in reaches],
                 sponge=sponge)
    total = sum(B.target)
    while B.active:
        if cancel and cancel():
            return results
        B.advance(400)
        if progress:
            first = next((i for i in B.active if i >= len(levels_used)), None)
            label = cases[first - len(levels_used)][2]["label"] if first is not None else test["title"]
            progress(sum(B.steps_done) / total, label)
    base_res = {h: profiles_device(B.runs[i]) for i, h in enumerate(levels_used)}
    for k, (h, rr, v) in enumerate(cases):
        run = B.runs[len(levels_used) + k]
        results.append(_result(profiles_device(run), base_res[h], rr, cfg, v))
        if on_result:
            on_result(results[-1], run)
    return results


def _result(res, base, reach, cfg, v):
    c = compare(res, base, reach, cfg)
    c["label"] = v["label"]
    c["profiles"] = res
    c["base_profiles"] = base
    c["notes"] = reach.notes
    return c
