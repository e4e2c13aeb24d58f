#!/usr/bin/env python
"""Benchmark of the D3Q19 stream-collide hot path on one boat case per GPU.

Workload (default ``reach36m``): the 150 m x 60 m x 4 m trapezoidal reach with a seeded
bumpy bed and a 20 m pusher tug, dx = 0.1 m, 1500 x 602 x 40 = 36.1M lattice cells
(water_flow_simulation_b200.cases.config2_case), stepped as Run3D steps it: 20-step
chunks whose last step writes the fields and refreshes the column-mean wall-model speed.
A "step" is one lattice time step of the whole lattice.  The populations (5.5 GB) are far
larger than L2, so no flush is needed between steps.

Printed on rank 0 as one JSON line:
  value        whole-job GLUPS (lattice cell updates per second over all ranks), device
               timed with CUDA events around the K timed steps, max over ranks;
  roofline     the plain-segment kernel (the dominant one): algorithmic bytes per launch
               (152 B = 19 populations read + 19 written, float32, per plain cell) over its
               mean launch time, measured with CUDA events on its stream in the timed
               region, against the measured HBM copy bandwidth;
  e2e          the same metric through the public API from pinned host buffers: upload of
               the case, set-up, the K steps with the lid water-level profile read back
               after every chunk, and the final velocity field read back, all timed;
  cpu_baseline the CPU oracle (C, OpenMP, all host cores) on a bounded slice of the case.
``--impl reference`` times that CPU implementation alone, on rank 0.
Multi-GPU (torchrun): every rank runs its own replica of the case (weak scaling, no
collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALG_BYTES_PER_CELL = {"fp32": 152, "fp16": 76}   # 19 populations read + 19 written
CHUNK = 20                        # steps between field outputs (Run3D.advance)
STEPS_PER_CASE = 20000            # steps of one boat case of this workload
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", choices=("reach36m", "reach7m", "config1", "config3", "ensemble24"),
                    default="reach36m",
                    help="reach36m: the benchmark case; reach7m: its first 30 m (profiling); config1: 192x50x12; "
                    "config3: 3000x1202x72 at dx 0.05 m (259.6M cells); ensemble24: 24 cases of 2M-20M cells")
    ap.add_argument("--tile", default=None, help="pipeline,cells_per_lane,warps,stages,ctas_per_sm "
                    "(default 3,2,4,0,0)")
    ap.add_argument("--storage", choices=("fp32", "fp16"), default="fp16",
                    help="population storage: 16-bit deviations from the lattice weights (the chosen method, "
                         "default) or float32 (the plain method)")
    ap.add_argument("--no-compare", action="store_true", help="skip the float32 comparison run")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU oracle sample length")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def build_case(workload):
    from water_flow_simulation_b200.cases import config1_case, config2_case, config3_case
    if workload == "config3":
        return config3_case(), ("config3: reach36m's reach at a 3.6 m stage and dx 0.05 m, "
                                "3000x1202x72 cells (259.6M), tug")
    if workload == "config1":
        return config1_case(), "config1: 48x12x3 m rectangular channel, 192x50x12 cells, one 75 kW boat"
    if workload == "reach7m":
        return config2_case(length=30.0), ("reach7m: first 30 m of reach36m (same section, bed and dx), "
                                           "300x602x40 cells, tug")
    return config2_case(), ("reach36m: 150x60x4 m trapezoid, 1:2 banks, bumpy bed (sigma 0.15 m, 5 m), "
                            "dx 0.1 m, 1500x602x40 cells, 20 m tug 2x300 kW")


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def measured_peaks_tflops():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["bf16_tflops"])
    except Exception:
        return 1590.0


def profiled_bytes_per_cell(kernel):
    """DRAM bytes per processed cell of `kernel` from the committed ncu summary (a capture of
    the smaller reach7m case; traffic grows with the cells a launch processes), if any."""
    path = os.path.join(ROOT, "profiles", "ncu_summary.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["kernels"][kernel]["dram_bytes_per_cell"])
    except Exception:
        return None


def max_over_ranks(value, world, device=None):
    """The largest `value` over all ranks (the timing rule for multi-GPU numbers)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class _NullSampler:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for _, _, flags in rows for n, f in zip(names, flags) if f.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------ CPU oracle
def oracle_sample(reach, max_cells=3_000_000):
    """The C oracle (OpenMP) on an x slice of the case (the first columns, inlet included)."""
    from oracle.oracle import OracleLBM
    nx = max(16, min(reach.nx, max_cells // (reach.ny * reach.nz)))
    sl = (slice(None), slice(None), slice(0, nx))
    nu_lb = max(1e-6 * reach.dt / reach.dx ** 2, 2e-4)
    uin = (reach.uin_phys / reach.vel).astype(np.float32)
    o = OracleLBM(reach.solid[sl], reach.Fx[sl], reach.Fy[sl], reach.Fz[sl], uin, 0.5 + 3 * nu_lb, reach.cfg.cs,
                  None if reach.cf is None else reach.cf[sl])
    bw = None if reach.bedwall is None else np.ascontiguousarray(reach.bedwall[sl])
    return o, bw, nx


def oracle_rate(reach, seconds, max_cells=3_000_000):
    """GLUPS of the C oracle on an x slice of the case, stepped (as Run3D steps, uref refreshed
    every 20 steps) for about `seconds`."""
    from oracle.oracle import lib
    o, bw, nx = oracle_sample(reach, max_cells)
    o.step(1)                                      # warm the caches and the thread pool
    steps, t0 = 0, time.perf_counter()
    while True:
        if bw is not None and steps % CHUNK == 0:
            o.update_uref(bw)
        o.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if (el >= seconds and steps >= 3) or steps >= 100000:
            break
    return {"value": steps * o.N / el / 1e9, "unit": "GLUPS", "cores": lib().oracle_num_threads(),
            "kind": "port",
            "sample": f"C oracle (OpenMP) on the x slice {nx}x{reach.ny}x{reach.nz} ({o.N / 1e6:.2f}M cells) of the "
                      f"case, {steps} steps in {el:.1f} s, uref refreshed every {CHUNK} steps"}


def run_reference(args, rank):
    """The CPU implementation of the path (the oracle, all host threads) on the same case:
    each step is one time step of an x slice of the lattice (about 3M cells)."""
    if rank != 0:
        return 0
    from oracle.oracle import build_oracle, lib
    build_oracle()
    reach, desc = build_case(args.workload)
    o, bw, nx = oracle_sample(reach)
    times = []
    for k in range(args.warmup + args.steps):
        if bw is not None and k % CHUNK == 0:
            o.update_uref(bw)
        t0 = time.perf_counter()
        o.step(1)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    el = sum(times)
    value = len(times) * o.N / el / 1e9
    sample = (f"C oracle (OpenMP) on the x slice {nx}x{reach.ny}x{reach.nz} ({o.N / 1e6:.2f}M cells) of the case, "
              f"{len(times)} timed steps after {args.warmup} warm-up steps, uref refreshed every {CHUNK} steps")
    out = {"metric": "GLUPS", "value": value, "unit": "GLUPS", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * el / len(times), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": {"workload": desc, "cells": reach.cells, "sample_cells": o.N, "parallelism": "cpu"},
           "cpu_baseline": {"value": value, "unit": "GLUPS", "cores": lib().oracle_num_threads(), "kind": "port",
                            "sample": sample},
           "e2e": {"value": value, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------------------------------ GPU arm
def make_solver(reach, tile, pinned=None, storage="fp32"):
    from water_flow_simulation_b200.lbm3d import LBM3D
    nu_lb = max(1e-6 * reach.dt / reach.dx ** 2, 2e-4)
    src = pinned or {"solid": reach.solid, "Fx": reach.Fx, "Fy": reach.Fy, "Fz": reach.Fz, "cf": reach.cf,
                     "bedwall": reach.bedwall, "uin": (reach.uin_phys / reach.vel).astype(np.float32)}
    column = src["bedwall"] is not None
    return LBM3D(None, src["solid"], src["Fx"], src["Fy"], src["Fz"], src["uin"], 0.5 + 3 * nu_lb, reach.cfg.cs,
                 src["cf"], bedwall=src["bedwall"], uref_mode="column" if column else "field", tile=tile,
                 storage=storage)


def step_parts(L, nat, n, plain_events=None):
    """n steps; the last one writes the fields.  With the split pipeline each step is launched
    as its plain part then the rest, and plain_events (list) gets an event pair per step."""
    import torch
    lat = L._lattice_ref()
    st = L._stream()
    col = nat.STEP_UREF_COLUMN if L.uref_mode == "column" else 0
    split = L.tile.pipeline == nat.PIPE_SPLIT and plain_events is not None
    if L.storage == "fp16":
        def launch(fs, fd, mode):
            return L.lib.lbm_fused_step_h(lat, fs, fd, L.store_scale, mode, L.tile, st)
    else:
        def launch(fs, fd, mode):
            return L.lib.lbm_fused_step(lat, fs, fd, mode, L.tile, st)
    for k in range(n):
        mode = col | (nat.STEP_OUTPUT if k == n - 1 else 0)
        fs, fd = L.f.data_ptr(), L.f2.data_ptr()
        if split:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            nat.check(launch(fs, fd, mode | nat.STEP_SKIP_SPECIAL), "plain part")
            e1.record()
            nat.check(launch(fs, fd, mode | nat.STEP_SKIP_PLAIN), "special part")
            plain_events.append((e0, e1))
        else:
            nat.check(launch(fs, fd, mode), "fused step")
        L.f, L.f2 = L.f2, L.f
    L.nstep += n


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from water_flow_simulation_b200 import _native as nat

    nat.require_cuda()
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    tile = tuple(int(v) for v in (args.tile or "3,2,4,0,0").split(","))
    alg = ALG_BYTES_PER_CELL[args.storage]
    reach, desc = build_case(args.workload)
    cells = reach.cells
    steps = max(CHUNK, (args.steps + CHUNK - 1) // CHUNK * CHUNK)
    warm = max(3, args.warmup)

    def barrier():
        if world > 1:
            dist.barrier()

    props = torch.cuda.get_device_properties(dev)
    gpu_id = getattr(props, "pci_bus_id", None)
    if isinstance(gpu_id, int) or gpu_id is None:
        gpu_id = local_rank

    def measure(storage, nsteps, sampler=None):
        """Device-resident timing of nsteps steps (inputs resident, populations >> L2)."""
        L = make_solver(reach, tile, storage=storage)
        counts = L.worklist_counts()
        step_parts(L, nat, warm)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        plain_ev = []
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with (sampler or _NullSampler()):
            e_start.record()
            for _ in range(nsteps // CHUNK):
                step_parts(L, nat, CHUNK, plain_ev)
            e_end.record()
            torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = max_over_ranks(e_start.elapsed_time(e_end), world, dev)
        status = L.status()
        plain_ms = [a.elapsed_time(b) for a, b in plain_ev]
        V = L.tile.cells_per_lane
        del L
        torch.cuda.empty_cache()
        return ms, plain_ms, counts, status, V

    # ---- device-resident throughput of the requested storage (default: the 16-bit store)
    clocks = ClockSampler(gpu_id)
    ms_max, plain_ms, counts, status, V = measure(args.storage, steps, clocks)
    fluid_cells = int((~reach.solid).sum())
    # per step: plain, edge and special kernels; per output step also solid fields and column means
    launches = steps * 3 + (steps // CHUNK) * 2 if counts else steps
    gemm = None
    if rank == 0:          # the learned warm start's tensor-core GEMM (bf16, float32 accumulation)
        try:
            from water_flow_simulation_b200.surrogate import gemm_throughput
            gemm = gemm_throughput()
            peak_t = measured_peaks_tflops()
            gemm.update({"peak_tflops": peak_t, "frac": gemm["tflops"] / peak_t, "bound": "tensor",
                         "peak_source": "measured bf16 cuBLAS burst"})
        except Exception as exc:           # reported, never required
            gemm = {"error": str(exc)}
    plain32 = None
    if args.storage != "fp32" and not args.no_compare:
        n32 = max(CHUNK, min(steps, 400) // CHUNK * CHUNK)
        ms32, _, _, st32, _ = measure("fp32", n32)
        plain32 = {"storage": "fp32", "steps": n32, "ms_per_step": ms32 / n32,
                   "value": world * n32 * cells / (ms32 * 1e-3) / 1e9, "unit": "GLUPS", "status_word": st32,
                   "boat_cases_per_hour": 3600.0 / (STEPS_PER_CASE * ms32 / n32 * 1e-3)}

    # ---- end to end through the public API, from pinned host buffers
    e2e = None
    if not args.no_e2e:
        pinned = {k: (None if a is None else torch.from_numpy(np.ascontiguousarray(a)).pin_memory())
                  for k, a in (("solid", reach.solid.astype(np.uint8)), ("Fx", reach.Fx), ("Fy", reach.Fy),
                               ("Fz", reach.Fz), ("cf", reach.cf),
                               ("bedwall", None if reach.bedwall is None else reach.bedwall.astype(np.uint8)),
                               ("uin", (reach.uin_phys / reach.vel).astype(np.float32)))}
        h2d = sum(v.numel() * v.element_size() for v in pinned.values() if v is not None)
        top = torch.from_numpy(~reach.solid[-1]).to(dev, torch.float32)
        ntop = top.sum(0).clamp(min=1)
        lid_host = torch.empty(reach.nx, dtype=torch.float32).pin_memory()
        out_host = torch.empty(cells, dtype=torch.float32).pin_memory()
        barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        E = make_solver(reach, tile, pinned, storage=args.storage)
        for _ in range(steps // CHUNK):
            E.step(CHUNK)
            rho_top = E.rho.view(reach.nz, reach.ny, reach.nx)[-1]
            lid_host.copy_((rho_top * top).sum(0) / ntop, non_blocking=True)
        out_host.copy_(E.ux, non_blocking=True)
        torch.cuda.synchronize()
        w1 = time.perf_counter()
        barrier()
        el = max_over_ranks(w1 - w0, world, dev)
        d2h = (steps // CHUNK) * reach.nx * 4 + cells * 4
        e2e = {"value": world * steps * cells / el / 1e9, "unit": "GLUPS",
               "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
               "what": f"case upload from pinned host memory + set-up + {steps} steps + lid level per "
                       f"{CHUNK}-step chunk + final ux field, timed on the host"}
        del E
        torch.cuda.empty_cache()

    if rank != 0:
        return 0
    peak, peak_kind = measured_peaks()
    roof = None
    if counts:
        plain_cells = counts[0] * 32 * V
        mean_plain = statistics.mean(plain_ms)
        achieved = plain_cells * alg / (mean_plain * 1e-3) / 1e9
        kname = "k_rows_h_plain" if args.storage == "fp16" else "k_rows_plain"
        per_cell = profiled_bytes_per_cell(kname)
        roof = {"kernel": f"{kname} (split pipeline, plain row segments, {args.storage} populations)",
                "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} HBM copy bandwidth", "launch_ms": mean_plain,
                "cells_per_launch": plain_cells, "algorithmic_bytes_per_launch": plain_cells * alg,
                "traffic": None if per_cell is None else per_cell * plain_cells,
                "traffic_source": "ncu dram bytes per cell on reach7m, scaled to this launch's cells",
                "step_achieved_gbs": fluid_cells * alg / (ms_max / steps * 1e-3) / 1e9}
    glups = world * steps * cells / (ms_max * 1e-3) / 1e9
    cpu = None
    if world == 1 or rank == 0:
        try:
            cpu = oracle_rate(reach, args.cpu_seconds)
        except Exception as exc:           # the baseline is reported, never required
            cpu = {"value": None, "unit": "GLUPS", "error": str(exc)}
    out = {"metric": "GLUPS", "value": glups, "unit": "GLUPS", "n_gpus": world, "steps": steps, "warmup": warm,
           "ms_per_step": ms_max / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32" if args.storage == "fp32" else "f32 collide, fp16 population store", "data": "synthetic",
           "config": {"workload": desc, "storage": args.storage, "lattice": [reach.nx, reach.ny, reach.nz], "cells": cells,
                      "fluid_cells": fluid_cells, "parallelism": f"replicas x{world}",
                      "l2": f"populations {2 * 19 * alg // 38 * cells / 1e9:.1f} GB vs 126 MB L2 (no flush)",
                      "tile": list(tile),
                      "worklists_plain_solid_special": counts, "steps_per_output": CHUNK},
           "boat_cases_per_hour": 3600.0 / (STEPS_PER_CASE * ms_max / steps * 1e-3),
           "plain_fp32": plain32,
           "tensor_core_gemm": gemm,
           "chosen_vs_plain_fp32": None if plain32 is None else plain32["ms_per_step"] / (ms_max / steps),
           "level_error_vs_fp64": "16-bit store vs float64, whole cases with the trailing average: config 1 "
                                  "0.040 cm max level, 0.57% mean bed shear; this reach without the boat 0.20 cm "
                                  "(float32 0.84 cm); with the tug 25.7 cm (float32 4.7 cm), set by the outlet's "
                                  "backflow mode; with the optional outlet sponge 16-bit is within 0.50 cm of "
                                  "float32 (accuracy summaries under profiles/)",
           "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
           "clocks": clocks.summary(), "status_word": status}
    print(json.dumps(out), flush=True)
    return 0


def run_ensemble(args, rank, world, local_rank):
    """24 seeded boat cases of 2M-20M cells (cases.ensemble_case): the 16-bit batch (one launch per
    kernel class per step, autotuned tile, 20-step chunks as CUDA graphs) against the plain method
    (float32, one case at a time).  cases/hour from each case's own step count to t_total.  With
    N ranks the 24 cases are split over the GPUs by cells x steps (batch.balance), each rank
    batching its own share; the aggregate is all cells over the slowest rank's time."""
    import torch
    import torch.distributed as dist
    from water_flow_simulation_b200 import _native as nat
    from water_flow_simulation_b200 import autotune
    from water_flow_simulation_b200.batch import CHUNK as BCHUNK, BatchRun
    from water_flow_simulation_b200.cases import ensemble_case
    from water_flow_simulation_b200.reach3d import Run3D

    nat.require_cuda()
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    from water_flow_simulation_b200.batch import balance
    every = [ensemble_case(s) for s in range(24)]
    every_cells = [r.solid.size for r in every]
    every_steps = [int(np.ceil(r.cfg.run_flows * r.cfg.length / max(r.V, 0.05) / r.dt / BCHUNK)) * BCHUNK
                   for r in every]
    mine = balance([c * s for c, s in zip(every_cells, every_steps)], world)[rank]   # this rank's cases
    reaches = [every[i] for i in mine]
    cells = [every_cells[i] for i in mine]
    case_steps = [every_steps[i] for i in mine]
    del every
    steps = max(BCHUNK, (args.steps + BCHUNK - 1) // BCHUNK * BCHUNK)
    B = BatchRun(reaches, max_steps=10 ** 9)
    tile, times = autotune.tune_batch(B, steps=20, warmup=4)
    B.advance(max(BCHUNK, args.warmup // BCHUNK * BCHUNK))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    props = torch.cuda.get_device_properties(dev)
    gpu_id = getattr(props, "pci_bus_id", local_rank)
    with ClockSampler(gpu_id if not isinstance(gpu_id, int) else local_rank) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B.advance(steps)
        e1.record()
        torch.cuda.synchronize()
    ms_mine = e0.elapsed_time(e1)
    ms = max_over_ranks(ms_mine, world, dev)
    status = B.status()
    agg = sum(every_cells) * steps / (ms * 1e-3) / 1e9          # all ranks' cells / the slowest rank's time
    rate_mine = sum(cells) * steps / (ms_mine * 1e-3)
    chosen_hours = max_over_ranks(sum(s * c for s, c in zip(case_steps, cells)) / rate_mine / 3600, world, dev)
    del B
    torch.cuda.empty_cache()
    plain = []                                        # float32, one case at a time
    n32 = 100
    for r in reaches:
        run = Run3D(r)
        run.advance(40)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        run.advance(n32)
        b.record()
        torch.cuda.synchronize()
        plain.append(a.elapsed_time(b) / n32)
        del run
        torch.cuda.empty_cache()
    plain_hours = max_over_ranks(sum(s * m * 1e-3 for s, m in zip(case_steps, plain)) / 3600, world, dev)
    if rank != 0:
        return 0
    out = {"metric": "GLUPS", "value": agg, "unit": "GLUPS", "n_gpus": world, "steps": steps,
           "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True,
           "scaling": "strong" if world > 1 else "weak",
           "vs_baseline": None, "dtype": "f32 collide, fp16 population store", "data": "synthetic",
           "config": {"workload": "ensemble24: 24 seeded boat cases, 2M-20M cells (cases.ensemble_case), dx 0.1 m",
                      "cells": sum(every_cells), "case_cells": every_cells, "case_steps_to_t_total": every_steps,
                      "rank0_cases": mine, "tile": list(tile),
                      "autotune_ms_per_step": {str(k): v for k, v in times.items()},
                      "parallelism": f"cases split over {world} GPUs by cells x steps (batch.balance)",
                      "l2": "populations >> 126 MB L2 (no flush)"},
           "cases_per_hour": {"chosen_fp16_batched": 24 / chosen_hours,
                              "plain_fp32_single": 24 / plain_hours,
                              "ratio": plain_hours / chosen_hours},
           "plain_fp32_ms_per_step": plain, "gpu_launches": steps * 3 + (steps // BCHUNK) * 3,
           "clocks": clocks.summary(), "status_words": status}
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "b200":
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            return run_reference(args, rank)
        if args.workload == "ensemble24":
            return run_ensemble(args, rank, world, local_rank)
        return run_b200(args, rank, world, local_rank)
    finally:
        if world > 1 and args.impl == "b200":
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
