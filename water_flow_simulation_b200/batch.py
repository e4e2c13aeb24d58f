"""Batched boat cases: many reaches of uneven sizes advanced together on one GPU.

Replaces the one-case-at-a-time loop of the reference's boat tests
(floodsim/boat_tests.py:73-113, Run3D.run_to_end at floodsim/reach3d.py:455-467).
Every case is a Run3D with 16-bit population storage; the batch steps all of them together
over the work lists of every case concatenated (entries tagged with their case): by default
one launch per kernel class per step (lbm_batch_step_h), or, with persistent=True, each
20-step chunk -- the steps of Run3D.advance between two field outputs -- as ONE persistent
cooperative launch (lbm_batch_chunk_h: every CTA resident for the chunk, grid barriers
between the steps; measured 17 % slower on the 24-case ensemble, so not the default; the
autotuner times both); either way the chunk is captured once as a CUDA graph and replayed.
Per case, as Run3D.advance does: the smoothstep force ramp (a scalar of the case's
lattice descriptor, in device memory, updated between chunks), the time averages in the
trailing window (a case outside its window has no accumulator in its descriptor), and the
stop at t_total.  A case can also stop at convergence: the relative change of its
discharge sum (float64, on the device), sampled every `check_every` steps, between the means
of its last two windows of `window` samples below `tol` (window 1: consecutive samples), and,
with `level_tol_cm`, the window-mean lid water level changing by less than that anywhere.  Finished cases
leave the batch; the rest are re-batched (new lists, new graphs).  With `observe_only` a case
that meets the stop rule runs on to its target, and the step and the window-mean level at the
stop are kept, so one run measures both what the stop saves and how far its answer lies from
the full run's (`stop_study`).
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _native as nat
from .lbm3d import ctypes_ptr
from .reach3d import Run3D

CHUNK = Run3D.avg_every
CASE_SHIFT = 24


def run_to_end_steps(reach, chunk=400):
    """The step count at which Run3D.run_to_end(chunk=chunk) stops a case: whole `chunk`-step
    calls of advance, each adding 20-step chunks of dt to t, until t >= t_total (the same
    float sums as Run3D, so the same stop)."""
    t_total = reach.cfg.run_flows * reach.cfg.length / max(reach.V, 0.05)
    t, steps = 0.0, 0
    while t < t_total:
        k = 0
        while k < chunk:
            m = min(CHUNK, chunk - k)
            t = t + m * reach.dt
            k += m
        steps += chunk
    return steps


def balance(work, parts):
    """Split cases over `parts` GPUs by their work (cells x steps): largest first, each to the
    GPU with the least work so far (ties to the lowest index).  Returns one sorted index list
    per GPU; every GPU then runs its own BatchRun with no exchange between them."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(work)), key=lambda k: (-float(work[k]), k)):
        g = min(range(parts), key=lambda p: (load[p], p))
        out[g].append(i)
        load[g] += float(work[i])
    return [sorted(o) for o in out]


class BatchRun:
    """Cases (Reach objects) advanced as one batch with 16-bit storage."""

    def __init__(self, reaches, tile=(3, 2, 4, 0, 0), use_graphs=True, tol=None, check_every=500,
                 max_steps=None, device=None, window=1, level_tol_cm=None, sponge=None, observe_only=False,
                 persistent=False):
        import torch
        nat.require_cuda()
        self.torch = torch
        self.lib = nat.load()
        if tile[0] != nat.PIPE_SPLIT or tile[1] != 2:
            raise ValueError("batches run the split pipeline on 64-cell segments: tile (3, 2, warps, stages, ctas)")
        self.tile = nat.Tile(*tile)
        self.use_graphs = use_graphs
        # persistent: a chunk is ONE cooperative launch of all its steps (lbm_batch_chunk_h), else
        # one launch per kernel class per step (lbm_batch_step_h); the results are the same bit for bit
        self.persistent = bool(persistent)
        self._sync = torch.zeros(4, dtype=torch.int32, device=device if device is not None else "cuda")
        self.tol, self.check_every, self.window = tol, int(check_every), int(window)
        self.level_tol_cm = level_tol_cm
        if self.check_every % CHUNK:
            raise ValueError(f"check_every must be a multiple of {CHUNK}")
        self.device = device
        self.runs = [Run3D(r, tile=tuple(tile), storage="fp16", sponge=sponge) for r in reaches]   # sponge: optional outlet sponge
        for run in self.runs:
            if run.lbm.uref_mode != self.runs[0].lbm.uref_mode:
                raise ValueError("all cases of a batch need the same uref mode")
            nseg = (run.lbm.pitch + 63) // 64 * run.lbm.ny * run.lbm.nz
            if nseg >= 1 << CASE_SHIFT:
                raise ValueError("a case has more than 2^24 row segments")
        self.steps_done = [0] * len(self.runs)
        if max_steps is None or np.ndim(max_steps) == 0:
            self.target = [int(math.ceil(run.t_total / run.r.dt / CHUNK)) * CHUNK if max_steps is None
                           else int(max_steps) for run in self.runs]
        else:                                           # one step target per case
            self.target = [int(m) for m in max_steps]
            if len(self.target) != len(self.runs) or any(m % CHUNK for m in self.target):
                raise ValueError(f"max_steps: one multiple of {CHUNK} per case")
        self.flux = [None] * len(self.runs)
        self.samples = [[] for _ in self.runs]          # (step, discharge sum, lid level profile)
        self.converged = [False] * len(self.runs)
        self.steps_to_converge = [None] * len(self.runs)
        # observe_only: a case that meets the stop rule keeps running to its target; the step and
        # the window-mean level at that point are recorded (to compare the stop's answer with the
        # full run's)
        self.observe_only = bool(observe_only)
        self.level_at_stop = [None] * len(self.runs)
        self.active = [i for i in range(len(self.runs))]
        self.wall = 0.0
        self._graphs = {}
        self._rebatch()

    # ------------------------------------------------------------------ batch tables
    def _rebatch(self):
        torch = self.torch
        self._graphs = {}
        runs = [self.runs[i] for i in self.active]
        if not runs:
            return
        dev = runs[0].lbm.device
        K = len(runs)
        self._lat_host = (nat.Lattice * K)(*[r.lbm._lattice() for r in runs])
        self._lat_dev = torch.empty(ctypes.sizeof(self._lat_host), dtype=torch.uint8, device=dev)
        self._po_dev = torch.empty(K * self.lib.lbm_batch_pull_offsets_bytes(), dtype=torch.uint8, device=dev)
        self._scale = torch.tensor([r.lbm.store_scale for r in runs], dtype=torch.float32, device=dev)
        self._pop = [torch.tensor([r.lbm.f.data_ptr() for r in runs], dtype=torch.int64, device=dev),
                     torch.tensor([r.lbm.f2.data_ptr() for r in runs], dtype=torch.int64, device=dev)]
        lists = []
        for k in range(4):                  # plain, solid, special, edge
            parts = []
            for c, r in enumerate(runs):
                lst, counts, v = r.lbm._wl
                if counts[k]:
                    parts.append(lst[k][:counts[k]].to(torch.int64) + (c << CASE_SHIFT))
            cat = torch.cat(parts).to(torch.int32) if parts else torch.zeros(1, dtype=torch.int32, device=dev)
            lists.append((cat, sum(int(r.lbm._wl[1][k]) for r in runs)))
        self._lists = lists
        b = nat.Batch()
        b.count = K
        b.max_columns = max(r.lbm.ny * r.lbm.pitch for r in runs)
        b.max_rows = max(r.lbm.ny * r.lbm.nz for r in runs)
        b.lat, b.pull_offsets = self._lat_dev.data_ptr(), self._po_dev.data_ptr()
        b.scale = self._scale.data_ptr()
        b.pop0, b.pop1 = self._pop[0].data_ptr(), self._pop[1].data_ptr()
        b.rows_plain, b.rows_solid, b.rows_special, b.rows_edge = (lst.data_ptr() for lst, _ in lists)
        b.n_plain, b.n_solid, b.n_special, b.n_edge = (n for _, n in lists)
        self._batch = b
        self._runs = runs
        self._upload_lattices([False] * K)
        nat.check(self.lib.lbm_batch_init(ctypes.byref(b), self._stream()), "lbm_batch_init")

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream

    def _upload_lattices(self, accumulate):
        """Force ramp and averaging switches of every active case -> device descriptors."""
        for c, run in enumerate(self._runs):
            L = run.lbm._lattice()
            if not accumulate[c]:
                L.avg = None
            self._lat_host[c] = L
        host = self.torch.frombuffer(bytearray(bytes(self._lat_host)), dtype=self.torch.uint8)
        self._lat_dev.copy_(host, non_blocking=False)

    # ------------------------------------------------------------------ stepping
    def _chunk(self, accumulate_any):
        """One chunk: CHUNK steps of every active case, the last one writing the fields."""
        col = nat.STEP_UREF_COLUMN if self._runs[0].lbm.uref_mode == "column" else 0
        last = col | nat.STEP_OUTPUT | (nat.STEP_ACCUMULATE if accumulate_any else 0)
        ref = ctypes.byref(self._batch)
        st = self._stream()
        if self.persistent:
            nat.check(self.lib.lbm_batch_chunk_h(ref, 0, CHUNK, col, last, self._sync.data_ptr(), st),
                      "lbm_batch_chunk_h")
            return
        for k in range(CHUNK):
            nat.check(self.lib.lbm_batch_step_h(ref, k & 1, last if k == CHUNK - 1 else col, self.tile, st),
                      "lbm_batch_step_h")

    def _run_chunk(self, accumulate_any):
        torch = self.torch
        if not self.use_graphs:
            self._chunk(accumulate_any)
            return
        g = self._graphs.get(accumulate_any)
        if g is None:
            self._chunk(accumulate_any)                 # eager first pass (also a warm-up)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._chunk(accumulate_any)
            self._graphs[accumulate_any] = g
            return                                     # the capture itself did not execute the chunk
        g.replay()

    def advance(self, nsteps):
        """Up to nsteps steps (a multiple of 20) of every active case; returns False when none is left."""
        torch = self.torch
        if nsteps % CHUNK:
            raise ValueError(f"nsteps must be a multiple of {CHUNK}")
        t0 = time.time()
        for _ in range(nsteps // CHUNK):
            if not self.active:
                break
            acc = []
            for run in self._runs:
                if not run._ramp_done:
                    f = min(run.t / run.t_ramp, 1.0)
                    f = np.float32(f * f * (3 - 2 * f))
                    run.lbm.force_scale = float(f)
                    run._ramp_done = f >= 1.0
                acc.append(run.t + CHUNK * run.r.dt >= run.t_avg)
            for run, a in zip(self._runs, acc):
                if a and run.lbm._avg is None:
                    run.lbm.enable_averaging()
            self._upload_lattices(acc)
            self._run_chunk(any(acc))
            for c, i in enumerate(self.active):
                run = self.runs[i]
                run.t += CHUNK * run.r.dt
                run.lbm.nstep += CHUNK
                if acc[c]:
                    run.navg += 1
                    run.lbm.navg += 1
                self.steps_done[i] += CHUNK
            self._retire()
        torch.cuda.synchronize()
        self.wall += time.time() - t0
        return bool(self.active)

    def _retire(self):
        """Drop cases that reached t_total or converged; re-batch the rest."""
        done = []
        W = self.window
        for i in self.active:
            n = self.steps_done[i]
            if self.tol is not None and n % self.check_every == 0 and not self.converged[i]:
                s = self.runs[i].lbm.profile_sums(mean=False)
                q = float(s["q"].sum())
                level = s["top_drho"] / np.maximum(s["top_n"], 1.0)
                self.samples[i].append((n, q, level))
                smp = self.samples[i]
                if len(smp) >= 2 * W:            # window means of the discharge sum over W samples
                    a = np.mean([x[1] for x in smp[-W:]])
                    b = np.mean([x[1] for x in smp[-2 * W:-W]])
                    ok = abs(a - b) <= self.tol * max(abs(a), 1e-30)
                    if ok and self.level_tol_cm is not None:   # and of the lid level profile, in cm
                        la = np.mean([x[2] for x in smp[-W:]], axis=0)
                        lb = np.mean([x[2] for x in smp[-2 * W:-W]], axis=0)
                        r = self.runs[i].r
                        ok = 100.0 / 3.0 * r.vel ** 2 / 9.81 * float(np.abs(la - lb).max()) <= self.level_tol_cm
                    if ok:
                        self.converged[i] = True
                        self.steps_to_converge[i] = n
                        self.level_at_stop[i] = np.mean([x[2] for x in smp[-W:]], axis=0)
                        if not self.observe_only:
                            done.append(i)
                            continue
            if n >= self.target[i]:
                done.append(i)
        if done:
            self.active = [i for i in self.active if i not in done]
            self._rebatch()

    def run_to_end(self, chunk_steps=400):
        while self.advance(chunk_steps):
            pass

    # ------------------------------------------------------------------ results
    def window_level(self, i):
        """Mean lid level (rho - 1 of the top layer, per x, lattice units) over the case's last
        window of samples (the level answer of a converged case)."""
        smp = self.samples[i][-self.window:]
        return np.mean([x[2] for x in smp], axis=0) if smp else None

    def status(self):
        return [run.lbm.status() for run in self.runs]

    @property
    def cells(self):
        return sum(run.lbm.N for run in self.runs)


def stop_study(seeds=range(24), tol=5e-3, window=8, check_every=500, level_tol_cm=0.25, log=None, series=False):
    """What a convergence stop saves on the seeded ensemble (cases.ensemble_case) and what it
    costs in accuracy.  All cases run in one 16-bit BatchRun to the step at which
    Run3D.run_to_end stops them (floodsim/reach3d.py:455-467: t_total, one flow-through), with
    the stop rule observed on the way: every `check_every` steps the discharge sum and the lid
    level profile are sampled, and a case counts as converged once the means of its last two
    windows of `window` samples differ by less than `tol` (relative, discharge) and
    `level_tol_cm` (anywhere along the reach).  Per case: the steps to the stop and to t_total,
    and the stop's answer -- the lid level profile (referenced to the outlet) averaged over
    its last window -- against the full run's (the time average over the trailing 40 % of
    t_total), as the largest difference along the reach and as the difference of the upstream
    level drop that `compare` reports.  Cases/hour with and without the stop use the batch's
    own measured rate (cells x steps per second over the whole run)."""
    import torch
    from .cases import ensemble_case
    from .reach3d import G, profiles_device
    reaches = [ensemble_case(int(s)) for s in seeds]
    targets = [run_to_end_steps(r) for r in reaches]
    B = BatchRun(reaches, max_steps=targets, tol=tol, window=window, check_every=check_every,
                 level_tol_cm=level_tol_cm, observe_only=True)
    torch.cuda.synchronize()
    t0 = time.time()
    while B.advance(2000):
        if log:
            log(f"{sum(B.steps_done)} case-steps, {len(B.active)} active, "
                f"{sum(1 for c in B.converged if c)} met the stop rule")
    torch.cuda.synchronize()
    wall = time.time() - t0
    cells = [r.solid.size for r in reaches]
    work_full = sum(c * n for c, n in zip(cells, B.steps_done))
    rate = work_full / wall
    cases = []
    for i, r in enumerate(reaches):
        full = profiles_device(B.runs[i])["eta"]
        row = {"seed": int(list(seeds)[i]), "cells": int(cells[i]), "steps_full": int(B.steps_done[i]),
               "steps_stop": B.steps_to_converge[i], "status": int(B.runs[i].lbm.status())}
        if B.level_at_stop[i] is not None:
            lv = B.level_at_stop[i] / 3.0 * r.vel ** 2 / G
            eta = lv - lv[-1]
            x = r.x
            i_up = max(int(0.08 * len(x)), 1)
            if r.hulls:
                i_up = max(min(i_up, int(np.searchsorted(x, min(hb[0] for hb in r.hulls) - 10.0))), 1)
            row["level_max_diff_cm"] = 100 * float(np.abs(eta - full).max())
            row["drop_diff_cm"] = 100 * float(abs((eta[i_up] - eta[-1]) - (full[i_up] - full[-1])))
        if series:                       # the sampled discharge and level (8 stations, cm, outlet-referenced)
            st = np.linspace(0, r.nx - 1, 8).astype(int)
            conv = 100.0 / 3.0 * r.vel ** 2 / G
            row["series"] = [[int(n), float(q)] + [round(conv * float(lv[k] - lv[-1]), 4) for k in st]
                             for n, q, lv in B.samples[i]]
            row["full_eta_cm"] = [round(100 * float(full[k]), 4) for k in st]
        cases.append(row)
    steps_stop = [c["steps_stop"] if c["steps_stop"] is not None else c["steps_full"] for c in cases]
    work_stop = sum(c * n for c, n in zip(cells, steps_stop))
    return {"seeds": [int(s) for s in seeds], "tol": tol, "window": window, "check_every": check_every,
            "level_tol_cm": level_tol_cm, "wall_s": wall, "glups": rate / 1e9,
            "cases_per_hour_full": len(reaches) * 3600 * rate / work_full,
            "cases_per_hour_stop": len(reaches) * 3600 * rate / work_stop,
            "stopped": sum(1 for c in cases if c["steps_stop"] is not None), "cases": cases}


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="convergence-stop study of the seeded ensemble")
    ap.add_argument("--cases", type=int, default=24)
    ap.add_argument("--tol", type=float, default=5e-3)
    ap.add_argument("--window", type=int, default=8)
    ap.add_argument("--check-every", type=int, default=500)
    ap.add_argument("--level-tol-cm", type=float, default=0.25)
    ap.add_argument("--out", default=None, help="JSON path for the result")
    ap.add_argument("--series", action="store_true", help="keep every case's sampled discharge and level")
    a = ap.parse_args(argv)
    res = stop_study(range(a.cases), a.tol, a.window, a.check_every, a.level_tol_cm,
                     log=lambda m: print(m, flush=True), series=a.series)
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
