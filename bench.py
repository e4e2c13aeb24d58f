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
               (76 B = 19 populations read + 19 written, 16-bit, per plain cell) over its
               mean launch time, measured with CUDA events on its stream in the timed
               region, against the measured HBM copy bandwidth;
  e2e          the same metric through the public API from pinned host buffers: upload of
               the case, set-up, the K steps with the lid water-level profile read back
               after every chunk, and the final velocity field read back, all timed;
  plain_fp32   the plain method (float32 populations) on the same case, with its own
               autotuned tile and its own plain-kernel roofline (152 B per plain cell);
  cpu_baseline the CPU restatement of the reference's Numba step, compiled in the reference's
               fast-math mode, OpenMP on all host cores, on the whole lattice (or an x slice
               when that would not fit the sample's few seconds);
  clocks       NVML samples of the SM clock and clock-event reasons over the timed steps and a
               following window of at least 1 s of the same steps.
Tiles come from the project's autotuner (autotune.tune_single) unless --tile is given.
``--impl reference`` times the CPU implementation alone, on rank 0.
Multi-GPU (torchrun): every rank runs its own replica of the case (weak scaling, no
collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
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
                    "(default: autotuned per storage)")
    ap.add_argument("--storage", choices=("fp32", "fp16"), default="fp16",
                    help="population storage: 16-bit deviations from the lattice weights (the chosen method, "
                         "default) or float32 (the plain method)")
    ap.add_argument("--no-compare", action="store_true", help="skip the float32 comparison run")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline sample length (about)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="profiling runs: only the device-timed passes (no float32 leg, GEMM, end-to-end, CPU "
                         "baseline or clock window)")
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
    """SM clock, power and clock-event reasons of this rank's GPU, polled through NVML every
    2 ms by a thread while active (the GPU is found by its UUID, so CUDA_VISIBLE_DEVICES
    cannot point it at another GPU).  It can be entered several times; samples taken while
    `region` is set are counted as the timed region's."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, uuid):
        self.uuid = uuid
        self.rows = []           # (in_region, sm_mhz, max_mhz, power_w, reason bits)
        self.region = False
        self.error = None
        self._stop = None
        self.nv = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid.encode() if isinstance(uuid, str) else uuid)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.bits = {n: int(getattr(pynvml, c, 0)) for n, c in self.REASONS}
        except Exception as exc:           # reported, never required
            self.error = f"NVML: {exc}"
            self.nv = None

    def _poll(self):
        nv, h = self.nv, self.h
        while not self._stop.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                reasons = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                power = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append((self.region, mhz, self.max_mhz, power, reasons))
            except Exception as exc:
                self.error = f"NVML: {exc}"
                return
            self._stop.wait(0.002)

    def __enter__(self):
        if self.nv is not None:
            self._stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        return self

    def __exit__(self, *exc):
        if self._stop is not None:
            self._stop.set()
            self.thread.join(timeout=2)
            self._stop = None
        return False

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"],
                    "error": self.error or "no samples"}
        reasons = sorted({n for *_, r in self.rows for n, b in self.bits.items() if b and r & b})
        timed = [r for r in self.rows if r[0]]
        return {"sm_mhz": statistics.median(r[1] for r in self.rows), "sm_max_mhz": max(r[2] for r in self.rows),
                "sm_mhz_min": min(r[1] for r in self.rows), "power_w_max": max(r[3] for r in self.rows),
                "reasons": reasons, "samples": len(self.rows), "samples_in_timed_region": len(timed),
                "sm_mhz_timed_region": statistics.median(r[1] for r in timed) if timed else None,
                "source": "NVML every 2 ms over the timed region and a following window of at least 1 s "
                          "of the same steps"}


def gpu_uuid(dev):
    import torch
    u = str(torch.cuda.get_device_properties(dev).uuid)
    return u if u.startswith("GPU-") else "GPU-" + u


# ------------------------------------------------------------------------------ CPU oracle
CPU_FULL_LATTICE_BUDGET_S = 150.0     # the whole lattice is stepped when warm-up + steps fit in this


def _cpu_lib():
    """The CPU restatement compiled as the reference compiles its CPU path (-O3 for this host,
    fast math), built here on the host it runs on (oracle.build_oracle_timing)."""
    import tempfile
    from oracle.oracle import timing_lib
    return timing_lib(os.path.join(tempfile.gettempdir(), f"lbm_oracle_timing_{os.getpid()}"))


def oracle_case(reach, clib, x_cols=None):
    """The CPU solver on the whole case, or on its first x_cols columns (inlet included)."""
    from oracle.oracle import OracleLBM
    nx = reach.nx if x_cols is None else max(16, min(reach.nx, x_cols))
    sl = (slice(None), slice(None), slice(0, nx))
    nu_lb = max(1e-6 * reach.dt / reach.dx ** 2, 2e-4)
    uin = (reach.uin_phys / reach.vel).astype(np.float32)
    o = OracleLBM(reach.solid[sl], reach.Fx[sl], reach.Fy[sl], reach.Fz[sl], uin, 0.5 + 3 * nu_lb, reach.cfg.cs,
                  None if reach.cf is None else reach.cf[sl], clib=clib)
    bw = None if reach.bedwall is None else np.ascontiguousarray(reach.bedwall[sl])
    return o, bw, nx


def cpu_steps(reach, n_steps, n_warm, budget_s=CPU_FULL_LATTICE_BUDGET_S):
    """Time n_steps CPU steps after n_warm (uref refreshed every 20 steps, as Run3D steps):
    on the whole lattice when one step, measured first on it, lets warm-up + steps fit in
    budget_s, else on an x slice of the lattice sized to fit.  Returns (per-step seconds,
    cells per step, description of the sample, threads)."""
    clib = _cpu_lib()
    o, bw, nx = oracle_case(reach, clib)
    if bw is not None:
        o.update_uref(bw)
    t0 = time.perf_counter()
    o.step(1)
    one = time.perf_counter() - t0
    if (n_steps + n_warm) * one > budget_s:
        cols = max(16, int(reach.nx * budget_s / ((n_steps + n_warm + 1) * one)))
        del o
        o, bw, nx = oracle_case(reach, clib, cols)
        o.step(1)
    times = []
    for k in range(n_warm + n_steps):
        if bw is not None and k % CHUNK == 0:
            o.update_uref(bw)
        t0 = time.perf_counter()
        o.step(1)
        if k >= n_warm:
            times.append(time.perf_counter() - t0)
    whole = nx == reach.nx
    what = ("the whole lattice" if whole else f"the x slice {nx}x{reach.ny}x{reach.nz} ({o.N / 1e6:.2f}M cells)")
    desc = (f"CPU restatement of floodsim's Numba step (oracle/lbm_oracle.c compiled -O3 -march=native "
            f"-ffast-math, the reference's fastmath=True mode; OpenMP, {clib.oracle_num_threads()} threads) on "
            f"{what}, {len(times)} timed steps after {n_warm} warm-up steps, uref refreshed every {CHUNK} steps")
    return times, o.N, desc, clib.oracle_num_threads(), whole


def run_reference(args, rank):
    """The CPU implementation of the path on the host cores, on the same case: each step is
    one time step of the whole lattice (or, when that would not fit a few minutes, of an x
    slice of it)."""
    if rank != 0:
        return 0
    reach, desc = build_case(args.workload)
    warm = max(3, args.warmup)
    times, n_cells, sample, cores, whole = cpu_steps(reach, args.steps, warm)
    el = sum(times)
    value = len(times) * n_cells / el / 1e9
    out = {"metric": "GLUPS", "value": value, "unit": "GLUPS", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": warm, "ms_per_step": 1e3 * el / len(times), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
           "config": {"workload": desc, "cells": reach.cells, "sample_cells": n_cells, "whole_lattice": whole,
                      "parallelism": "cpu"},
           "cpu_baseline": {"value": value, "unit": "GLUPS", "cores": cores, "kind": "port", "sample": sample},
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
    """n steps; the last one writes the fields.  With the split pipeline and plain_events (a list)
    each step is launched as its plain part then the rest, and plain_events gets an event pair
    per step; without, a step is one call (overlapped when the solver's tile says so)."""
    import torch
    lat = L._lattice_ref()
    st = L._stream()
    col = nat.STEP_UREF_COLUMN if L.uref_mode == "column" else 0
    split = L.tile.pipeline == nat.PIPE_SPLIT and plain_events is not None
    if L.overlap and L.tile.pipeline == nat.PIPE_SPLIT and not split:
        col |= nat.STEP_OVERLAP
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


def plain_roofline(storage, counts, V, plain_ms, peak, peak_kind, fluid_cells, step_ms):
    """Roofline of the plain-segment kernel: its algorithmic bytes per launch (19 populations
    read + 19 written per plain cell) over its mean launch time (CUDA events around it on its
    stream, in every step of a second timed pass whose steps launch the plain kernel apart from
    the rest), against the HBM copy bandwidth; step_* give the whole step of the first pass."""
    alg = ALG_BYTES_PER_CELL[storage]
    plain_cells = counts[0] * 32 * V
    mean_plain = statistics.mean(plain_ms)
    achieved = plain_cells * alg / (mean_plain * 1e-3) / 1e9
    kname = "k_rows_h_plain" if storage == "fp16" else "k_rows_plain"
    per_cell = profiled_bytes_per_cell(kname)
    return {"kernel": f"{kname} (split pipeline, plain row segments, {storage} populations)", "bound": "hbm",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": f"{peak_kind} HBM copy bandwidth", "launch_ms": mean_plain, "launches": len(plain_ms),
            "cells_per_launch": plain_cells, "algorithmic_bytes_per_cell": alg,
            "algorithmic_bytes_per_launch": plain_cells * alg,
            "traffic": None if per_cell is None else per_cell * plain_cells,
            "traffic_source": "ncu dram bytes per cell on reach7m, scaled to this launch's cells",
            "step_achieved_gbs": fluid_cells * alg / (step_ms * 1e-3) / 1e9,
            "step_frac": fluid_cells * alg / (step_ms * 1e-3) / 1e9 / peak}


def accuracy_statement():
    """The measured accuracy of this workload against float64, from the committed statement
    (profiles/accuracy_statement_reach36m.json, written by
    `python -m water_flow_simulation_b200.accuracy --statement ...`): for each storage, the
    boat run's largest time-averaged level difference and the error of the boat's level change,
    beside the float64 floor (float64 from a start perturbed by half a float32 ulp); or None."""
    path = os.path.join(ROOT, "profiles", "accuracy_statement_reach36m.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
    except Exception:
        return None
    boat, lc = d["boat"], d["level_change"]
    out = {"source": "profiles/accuracy_statement_reach36m.json", "steps": d["steps"],
           "averaged_from_step": d["avg_from"], "fp64_level_change_cm": lc["fp64"]["d_eta_cm"]}
    for k in ("fp64p", "fp32", "fp16"):
        name = "fp64_floor" if k == "fp64p" else k
        out[name] = {"level_max_cm": boat[k]["level_max_cm"], "level_change_error_cm": lc[k]["error_cm"],
                     "shear_max_rel": boat[k]["shear_max_rel"]}
        if "shear_avg_rel" in boat[k]:
            out[name]["shear_avg_rel"] = boat[k]["shear_avg_rel"]
        eff = d.get("boat_effects", {}).get(k)
        if eff:
            out[name]["discharge_gain_error_pct"] = eff["error"]["dQ_net_pct"]
    if "fp64" in d.get("boat_effects", {}):
        out["fp64_discharge_gain_pct"] = d["boat_effects"]["fp64"]["dQ_net_pct"]
    return out


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from water_flow_simulation_b200 import _native as nat
    from water_flow_simulation_b200 import autotune

    nat.require_cuda()
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    fixed_tile = None if not args.tile else tuple(int(v) for v in args.tile.split(","))
    reach, desc = build_case(args.workload)
    cells = reach.cells
    steps = max(CHUNK, (args.steps + CHUNK - 1) // CHUNK * CHUNK)
    warm = max(3, args.warmup)
    fluid_cells = int((~reach.solid).sum())

    def barrier():
        if world > 1:
            dist.barrier()

    clocks = ClockSampler(gpu_uuid(dev))

    def measure(storage, nsteps, sampler=None):
        """Device-resident timing of nsteps steps (inputs resident, populations >> L2), with the
        tile the autotuner picks for this lattice (or --tile).  With a sampler, the clocks are
        sampled over the timed steps and over a following window of at least 1 s of the same
        steps (not part of the timed number)."""
        L = make_solver(reach, fixed_tile or (3, 2, 4, 0, 0), storage=storage)
        tune_ms = {}
        if fixed_tile is None:
            tile, tune_ms = autotune.tune_single(L, steps=20, warmup=4)
        counts = L.worklist_counts()
        step_parts(L, nat, warm)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with (sampler or _NullSampler()):
            if sampler is not None:
                sampler.region = True
            e_start.record()
            for _ in range(nsteps // CHUNK):
                step_parts(L, nat, CHUNK)
            e_end.record()
            torch.cuda.synchronize()
            if sampler is not None:
                sampler.region = False
                t0 = time.perf_counter()
                while time.perf_counter() - t0 < 1.0:
                    step_parts(L, nat, CHUNK)
                    torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ms = max_over_ranks(e_start.elapsed_time(e_end), world, dev)
        # the dominant kernel alone: the same number of steps again, each launched as its plain
        # part then the rest (no overlap), with CUDA events around every plain launch
        plain_ev = []
        k_start, k_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k_start.record()
        for _ in range(nsteps // CHUNK):
            step_parts(L, nat, CHUNK, plain_ev)
        k_end.record()
        torch.cuda.synchronize()
        split_ms = k_start.elapsed_time(k_end)
        status = L.status()
        plain_ms = [a.elapsed_time(b) for a, b in plain_ev]
        tile = L.tile_key()
        V = L.tile.cells_per_lane
        del L
        torch.cuda.empty_cache()
        return dict(ms=ms, plain_ms=plain_ms, counts=counts, status=status, V=V, tile=list(tile),
                    split_ms_per_step=split_ms / nsteps,
                    autotune_ms_per_step={",".join(map(str, k)): v for k, v in tune_ms.items()})

    # ---- device-resident throughput of the requested storage (default: the 16-bit store)
    if args.quick:
        args.no_compare = args.no_e2e = True
    main = measure(args.storage, steps, None if args.quick else clocks)
    ms_max = main["ms"]
    counts = main["counts"]
    # per step: plain, edge and special kernels; per output step also solid fields and column means
    launches = steps * 3 + (steps // CHUNK) * 2 if counts else steps
    gemm = None
    if rank == 0 and not args.quick:   # the learned warm start's tensor-core GEMM (bf16, float32 accumulation)
        try:
            from water_flow_simulation_b200.surrogate import gemm_throughput
            gemm = gemm_throughput()
            peak_t = measured_peaks_tflops()
            gemm.update({"peak_tflops": peak_t, "frac": gemm["tflops"] / peak_t, "bound": "tensor",
                         "peak_source": "measured bf16 cuBLAS burst"})
        except Exception as exc:           # reported, never required
            gemm = {"error": str(exc)}
    peak, peak_kind = measured_peaks()
    plain32 = None
    if args.storage != "fp32" and not args.no_compare:
        n32 = max(CHUNK, min(steps, 400) // CHUNK * CHUNK)
        m32 = measure("fp32", n32)
        plain32 = {"storage": "fp32", "steps": n32, "ms_per_step": m32["ms"] / n32,
                   "value": world * n32 * cells / (m32["ms"] * 1e-3) / 1e9, "unit": "GLUPS",
                   "status_word": m32["status"], "tile": m32["tile"],
                   "autotune_ms_per_step": m32["autotune_ms_per_step"],
                   "boat_cases_per_hour": 3600.0 / (STEPS_PER_CASE * m32["ms"] / n32 * 1e-3),
                   "roofline": None if not m32["counts"] else plain_roofline(
                       "fp32", m32["counts"], m32["V"], m32["plain_ms"], peak, peak_kind, fluid_cells,
                       m32["ms"] / n32)}

    # ---- end to end through the public API, from pinned host buffers
    e2e = None
    if not args.no_e2e:
        tile = tuple(main["tile"])
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
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

        def e2e_pass():
            """One case through the public API: upload + set-up, the steps with the lid level read
            back per chunk, the final ux field read back; host clock around it, CUDA events at
            the phase boundaries."""
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ev[0].record()
            E = make_solver(reach, tile, pinned, storage=args.storage)
            ev[1].record()
            chunk_ev = []
            for _ in range(steps // CHUNK):
                E.step(CHUNK)
                chunk_ev.append(torch.cuda.Event(enable_timing=True))
                chunk_ev[-1].record()
                lid_host.copy_((E.layer("rho", -1) * top).sum(0) / ntop, non_blocking=True)
            ev[2].record()
            out_host.copy_(E.ux, non_blocking=True)
            ev[3].record()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            barrier()
            del E
            return t0, t1, chunk_ev

        # one untimed pass first: it pays the process's one-off costs -- CUDA's lazy loading of
        # the library and torch kernels the readouts use first here (14.5 ms measured), the first
        # DMA into the newly pinned buffers (a few to hundreds of ms between boxes) -- which a
        # process running case after case pays once, not per case
        e2e_pass()
        w0, w1, chunk_ev = e2e_pass()
        el = max_over_ranks(w1 - w0, world, dev)
        d2h = (steps // CHUNK) * reach.nx * 4 + cells * 4
        e2e = {"value": world * steps * cells / el / 1e9, "unit": "GLUPS",
               "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
               "what": f"case upload from pinned host memory + set-up + {steps} steps + lid level per "
                       f"{CHUNK}-step chunk + final ux field, timed on the host, after one untimed pass "
                       f"of the same sequence (process warm-up)",
               "phases_ms": {"upload_and_setup": ev[0].elapsed_time(ev[1]),
                             "steps_and_lid_levels": ev[1].elapsed_time(ev[2]),
                             "first_chunk_steps": ev[1].elapsed_time(chunk_ev[0]),
                             "ux_readback": ev[2].elapsed_time(ev[3]),
                             "host_total": (w1 - w0) * 1e3,
                             "note": "CUDA events on the stream (no added synchronisation); host_total "
                                     "also holds the host's own work between launches"}}
        torch.cuda.empty_cache()

    if rank != 0:
        return 0
    roof = None
    if counts:
        roof = plain_roofline(args.storage, counts, main["V"], main["plain_ms"], peak, peak_kind, fluid_cells,
                              ms_max / steps)
    glups = world * steps * cells / (ms_max * 1e-3) / 1e9
    cpu = None
    try:
        if args.quick:
            raise RuntimeError("skipped (--quick)")
        n_cpu = max(3, int(args.cpu_seconds))
        times, n_cells, sample, cores, whole = cpu_steps(reach, n_cpu, 1, budget_s=3 * args.cpu_seconds)
        cpu = {"value": len(times) * n_cells / sum(times) / 1e9, "unit": "GLUPS", "cores": cores, "kind": "port",
               "sample": sample, "whole_lattice": whole}
    except Exception as exc:           # the baseline is reported, never required
        cpu = {"value": None, "unit": "GLUPS", "error": str(exc)}
    acc = accuracy_statement()
    out = {"metric": "GLUPS", "value": glups, "unit": "GLUPS", "n_gpus": world, "steps": steps, "warmup": warm,
           "ms_per_step": ms_max / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32" if args.storage == "fp32" else "f32 collide, fp16 population store", "data": "synthetic",
           "config": {"workload": desc, "storage": args.storage, "lattice": [reach.nx, reach.ny, reach.nz],
                      "cells": cells, "fluid_cells": fluid_cells, "parallelism": f"replicas x{world}",
                      "l2": f"populations {2 * 19 * ALG_BYTES_PER_CELL[args.storage] // 38 * cells / 1e9:.1f} GB "
                            f"vs 126 MB L2 (no flush)",
                      "tile": main["tile"], "tile_source": "--tile" if fixed_tile else "autotune.tune_single",
                      "autotune_ms_per_step": main["autotune_ms_per_step"],
                      "worklists_plain_solid_special_edge": counts, "steps_per_output": CHUNK,
                      "roofline_pass_ms_per_step": main["split_ms_per_step"]},
           "boat_cases_per_hour": 3600.0 / (STEPS_PER_CASE * ms_max / steps * 1e-3),
           "plain_fp32": plain32,
           "tensor_core_gemm": gemm,
           "chosen_vs_plain_fp32": None if plain32 is None else plain32["ms_per_step"] / (ms_max / steps),
           "level_error_vs_fp64": acc,
           "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
           "clocks": clocks.summary(), "status_word": main["status"]}
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
    clocks = ClockSampler(gpu_uuid(dev))
    with clocks:
        clocks.region = True
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        B.advance(steps)
        e1.record()
        torch.cuda.synchronize()
        clocks.region = False
    ms_mine = e0.elapsed_time(e1)
    ms = max_over_ranks(ms_mine, world, dev)
    status = B.status()
    agg = sum(every_cells) * steps / (ms * 1e-3) / 1e9          # all ranks' cells / the slowest rank's time
    rate_mine = sum(cells) * steps / (ms_mine * 1e-3)
    chosen_hours = max_over_ranks(sum(s * c for s, c in zip(case_steps, cells)) / rate_mine / 3600, world, dev)
    del B
    torch.cuda.empty_cache()
    plain, single16 = [], []          # float32 one case at a time; the 16-bit store one case at a time
    n32 = 100
    for r in reaches:
        for storage, acc in (("fp32", plain), ("fp16", single16)):
            run = Run3D(r, storage=storage)
            run.advance(40)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            run.advance(n32)
            b.record()
            torch.cuda.synchronize()
            acc.append(a.elapsed_time(b) / n32)
            del run
            torch.cuda.empty_cache()
    plain_hours = max_over_ranks(sum(s * m * 1e-3 for s, m in zip(case_steps, plain)) / 3600, world, dev)
    single16_hours = max_over_ranks(sum(s * m * 1e-3 for s, m in zip(case_steps, single16)) / 3600, world, dev)
    single16_glups = sum(cells) / (sum(single16) * 1e-3) / 1e9
    if rank != 0:
        return 0
    out = {"metric": "GLUPS", "value": agg, "unit": "GLUPS", "n_gpus": world, "steps": steps,
           "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True,
           "scaling": "strong" if world > 1 else "weak",
           "vs_baseline": None, "dtype": "f32 collide, fp16 population store", "data": "synthetic",
           "config": {"workload": "ensemble24: 24 seeded boat cases, 2M-20M cells (cases.ensemble_case), dx 0.1 m",
                      "cells": sum(every_cells), "case_cells": every_cells, "case_steps_to_t_total": every_steps,
                      "rank0_cases": mine, "tile": tile if isinstance(tile, str) else list(tile),
                      "autotune_ms_per_step": {str(k): v for k, v in times.items()},
                      "parallelism": f"cases split over {world} GPUs by cells x steps (batch.balance)",
                      "l2": "populations >> 126 MB L2 (no flush)"},
           "cases_per_hour": {"chosen_fp16_batched": 24 / chosen_hours,
                              "plain_fp32_single": 24 / plain_hours,
                              "fp16_single": 24 / single16_hours,
                              "ratio": plain_hours / chosen_hours,
                              "batching_gain_over_fp16_single": single16_hours / chosen_hours},
           "fp16_single_glups_same_cases": single16_glups,
           "plain_fp32_ms_per_step": plain, "fp16_single_ms_per_step": single16,
           "gpu_launches": (steps // BCHUNK) if tile == "persistent" else steps * 3 + (steps // BCHUNK) * 3,
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
