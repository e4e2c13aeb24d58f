"""Tile autotuner for the fused step: times candidate launch shapes on the real lattice.

A candidate is an lbm_tile (pipeline, cells_per_lane, warps, stages, ctas_per_sm).  Each is
timed with CUDA events over a few steps of the caller's own case (or batch) after a warm-up,
on the same stream, and the fastest wins.  Results are cached per lattice signature
(storage, shape, work-list sizes) in memory and, when `cache_path` is given, in a JSON file,
so a sweep of many similar cases tunes once.  Timing steps advance the state like any other
steps; tuning is done on a scratch copy of the populations, restored afterwards.
"""
from __future__ import annotations

import json
import os

from . import _native as nat

# candidates: the split pipeline is the fast family on every lattice measured; the
# register pipeline is kept as a reference point.  A sixth entry 1 runs the edge and special
# kernels beside the plain kernel (LBM3D.overlap), ctas_per_sm then bounding the plain kernel.
SINGLE_FP32 = [(3, 2, 4, 0, 0), (3, 2, 2, 0, 0), (3, 4, 4, 0, 0), (3, 2, 4, 0, 4), (3, 4, 2, 0, 0), (0, 2, 4, 0, 0),
               (3, 4, 4, 0, 0, 1), (3, 4, 4, 0, 2, 1), (3, 2, 4, 0, 2, 1)]
SINGLE_FP16 = [(3, 2, 4, 0, 0), (3, 2, 2, 0, 0), (3, 2, 4, 4, 0), (3, 4, 4, 0, 0), (3, 2, 4, 0, 2), (3, 8, 4, 0, 0),
               (3, 2, 4, 0, 0, 1), (3, 2, 4, 0, 2, 1), (3, 2, 4, 0, 1, 1)]
BATCH_FP16 = [(3, 2, 4, 0, 0), (3, 2, 2, 0, 0), (3, 2, 4, 4, 0), (3, 2, 4, 0, 2), (3, 2, 1, 0, 0)]

_memo: dict = {}


def _load(path):
    if path and os.path.exists(path):
        try:
            with open(path) as fh:
                return json.load(fh)
        except (OSError, ValueError):
            return {}
    return {}


def _save(path, data):
    if not path:
        return
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _time(torch, run_steps, steps, warmup):
    run_steps(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run_steps(steps)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def tune_single(L, candidates=None, steps=20, warmup=4, cache_path=None):
    """Pick the fastest tile for LBM3D `L`, set it, and return (tile, {tile: ms per step})."""
    torch = L._torch
    if candidates is None:
        candidates = SINGLE_FP16 if L.storage == "fp16" else SINGLE_FP32
    key = f"single/{L.storage}/{L.nx}x{L.ny}x{L.nz}"
    cache = _load(cache_path)
    if key in _memo or key in cache:
        best = tuple(_memo.get(key) or cache[key]["tile"])
        L.set_tile(best)
        return best, {}
    f0, f20 = L.f.clone(), L.f2.clone()
    fields = [t.clone() for t in (L._rho, L._ux, L._uy, L._uz, L._colU)]
    times = {}
    for tile in candidates:
        try:
            L.set_tile(tile)
        except nat.LBMError:
            continue

        def run_steps(n, L=L):
            k = 0
            while k < n:
                m = min(20, n - k)
                L.step(m)
                k += m
        try:
            times[tuple(tile)] = _time(torch, run_steps, steps, warmup)
        except nat.LBMError:
            continue
    best = min(times, key=times.get)
    L.f.copy_(f0)
    L.f2.copy_(f20)
    for t, s in zip((L._rho, L._ux, L._uy, L._uz, L._colU), fields):
        t.copy_(s)
    L.set_tile(best)
    _memo[key] = best
    cache[key] = {"tile": list(best), "ms_per_step": times[best]}
    _save(cache_path, cache)
    return best, times


def tune_batch(batch, candidates=None, steps=20, warmup=4, cache_path=None):
    """Pick the fastest way to step a BatchRun: one launch per kernel class per step with one of
    the candidate tiles (its cases' lists stay at 64-cell segments), or the whole 20-step chunk
    in one persistent launch (candidate "persistent").  Each is timed on whole chunks (the last
    step writing the fields), as BatchRun runs them; populations and fields are restored."""
    torch = batch.torch
    if candidates is None:
        candidates = BATCH_FP16 + ["persistent"]
    runs = [batch.runs[i] for i in batch.active]
    key = "batch/fp16/" + ",".join(f"{r.lbm.nx}x{r.lbm.ny}x{r.lbm.nz}" for r in runs)
    cache = _load(cache_path)
    if key in _memo or key in cache:
        best = _memo.get(key) or cache[key]["tile"]
        _apply_batch(batch, best)
        return (best if best == "persistent" else tuple(best)), {}
    saved = [(r.lbm.f.clone(), r.lbm.f2.clone()) for r in runs]
    fields = [[t.clone() for t in (r.lbm._rho, r.lbm._ux, r.lbm._uy, r.lbm._uz, r.lbm._colU)] for r in runs]
    chunks = max(1, steps // 20)
    times = {}
    for cand in candidates:
        _apply_batch(batch, cand)

        def run_steps(n):
            for _ in range(max(1, n // 20)):
                batch._chunk(False)
        try:
            ms = _time(torch, run_steps, 20 * chunks, max(20, warmup))
        except nat.LBMError:
            continue
        times[cand if cand == "persistent" else tuple(cand)] = ms
    for r, (a, b), fl in zip(runs, saved, fields):
        r.lbm.f.copy_(a)
        r.lbm.f2.copy_(b)
        for t, v in zip((r.lbm._rho, r.lbm._ux, r.lbm._uy, r.lbm._uz, r.lbm._colU), fl):
            t.copy_(v)
    best = min(times, key=times.get)
    _apply_batch(batch, best)
    _memo[key] = best
    cache[key] = {"tile": best if best == "persistent" else list(best), "ms_per_step": times[best]}
    _save(cache_path, cache)
    return best, times


def _apply_batch(batch, cand):
    """Set a BatchRun to a tune_batch candidate (a tile, or "persistent")."""
    if cand == "persistent":
        batch.persistent = True
    else:
        batch.persistent = False
        batch.tile = nat.Tile(*cand)
    batch._graphs = {}
