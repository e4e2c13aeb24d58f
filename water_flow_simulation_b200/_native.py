"""Build and load liblbm_b200.so (the sm_100a kernels) and describe its C ABI to ctypes.

The library is built in-tree by nvcc into ``water_flow_simulation_b200/_lib``.
There is no CPU fallback: if the library cannot be built or loaded, or no CUDA
device is present, every solver call raises.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(PKG, "_lib")
LIBNAME = "liblbm_b200.so"
LIBPATH = os.path.join(LIBDIR, LIBNAME)

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "--use_fast_math", "-Xcompiler", "-fPIC", "-shared"]

# flag and mode bits, mirrored from include/lbm_b200.h
FLAG_WALLS = 0x0007FFFE
FLAG_SOLID = 1 << 19
FLAG_FORCE = 1 << 20
FLAG_WALLFN = 1 << 21
FLAG_BEDWALL = 1 << 22
FLAG_GHOST = 1 << 23
STEP_OUTPUT = 1
STEP_UREF_COLUMN = 2
STEP_ACCUMULATE = 4
STEP_SKIP_PLAIN = 8
STEP_SKIP_SPECIAL = 16
STEP_OVERLAP = 32
PIPE_REGISTER = 0
PIPE_TMA = 1
PIPE_ASYNC = 2
PIPE_SPLIT = 3

LBM_OK = 0
ABI_VERSION = 113   # LBM_ABI_VERSION of include/lbm_b200.h


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return _sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))


def stale() -> bool:
    if not os.path.exists(LIBPATH):
        return True
    t = os.path.getmtime(LIBPATH)
    return any(os.path.getmtime(p) > t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu under csrc/ into one shared library for sm_100a."""
    if not force and not stale():
        return LIBPATH
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIBPATH + f".tmp{os.getpid()}"
    cmd = ["nvcc", *NVCC_FLAGS, "-I", INCLUDE, "-o", tmp, *_sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd)
    os.replace(tmp, LIBPATH)
    return LIBPATH


class Lattice(ctypes.Structure):
    """ctypes mirror of `lbm_lattice` (include/lbm_b200.h)."""
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("pitch", ctypes.c_int32),
                ("cells", ctypes.c_int64),
                ("tau0", ctypes.c_float), ("csmag2", ctypes.c_float), ("rho_out", ctypes.c_float),
                ("force_scale", ctypes.c_float),
                ("flags", ctypes.c_void_p), ("Fx", ctypes.c_void_p), ("Fy", ctypes.c_void_p), ("Fz", ctypes.c_void_p),
                ("cfw", ctypes.c_void_p), ("uref", ctypes.c_void_p), ("uin", ctypes.c_void_p),
                ("rho", ctypes.c_void_p), ("ux", ctypes.c_void_p), ("uy", ctypes.c_void_p), ("uz", ctypes.c_void_p),
                ("colU", ctypes.c_void_p), ("avg", ctypes.c_void_p), ("status", ctypes.c_void_p),
                ("rows_plain", ctypes.c_void_p), ("rows_solid", ctypes.c_void_p), ("rows_special", ctypes.c_void_p),
                ("n_plain", ctypes.c_int32), ("n_solid", ctypes.c_int32), ("n_special", ctypes.c_int32),
                ("list_cells_per_lane", ctypes.c_int32), ("rows_edge", ctypes.c_void_p), ("n_edge", ctypes.c_int32),
                ("sponge_cols", ctypes.c_int32), ("sponge_tau", ctypes.c_float), ("reserved", ctypes.c_int32)]


class Batch(ctypes.Structure):
    """ctypes mirror of `lbm_batch`."""
    _fields_ = [("count", ctypes.c_int32), ("max_columns", ctypes.c_int32), ("max_rows", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("lat", ctypes.c_void_p), ("pull_offsets", ctypes.c_void_p),
                ("scale", ctypes.c_void_p), ("pop0", ctypes.c_void_p), ("pop1", ctypes.c_void_p),
                ("rows_plain", ctypes.c_void_p), ("rows_solid", ctypes.c_void_p), ("rows_special", ctypes.c_void_p),
                ("rows_edge", ctypes.c_void_p), ("n_plain", ctypes.c_int32), ("n_solid", ctypes.c_int32),
                ("n_special", ctypes.c_int32), ("n_edge", ctypes.c_int32)]


class Tile(ctypes.Structure):
    """ctypes mirror of `lbm_tile`."""
    _fields_ = [("pipeline", ctypes.c_int32), ("cells_per_lane", ctypes.c_int32), ("warps", ctypes.c_int32),
                ("stages", ctypes.c_int32), ("ctas_per_sm", ctypes.c_int32)]

    def key(self):
        return (self.pipeline, self.cells_per_lane, self.warps, self.stages, self.ctas_per_sm)

    def __repr__(self):
        return ("Tile(pipeline={}, cells_per_lane={}, warps={}, stages={}, ctas_per_sm={})"
                .format(*self.key()))


# name -> (restype, argtypes); every exported symbol of include/lbm_b200.h
P, I32, U32, F32, F64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_float, ctypes.c_double
SIGNATURES = {
    "lbm_last_error": (ctypes.c_char_p, []),
    "lbm_abi_version": (I32, []),
    "lbm_device_sm_count": (I32, []),
    "lbm_step": (I32, [P] * 12 + [I32] * 3 + [F32, F32, P]),
    "lbm_bc": (I32, [P, P, P, I32, I32, I32, F32, P]),
    "lbm_export_blocks": (ctypes.c_int64, [ctypes.POINTER(Lattice)]),
    "lbm_export_velocity": (I32, [ctypes.POINTER(Lattice), I32, F32, P, P, P, P, P]),
    "lbm_move_particles": (I32, [ctypes.POINTER(Lattice), P, ctypes.c_int64, F32, F32, F64, P, I32,
                                 ctypes.c_uint64, ctypes.c_uint64, P, P]),
    "lbm_build_reach_masks": (I32, [I32, I32, I32, P, P, P, P, P, P, P]),
    "lbm_build_reach_walls": (I32, [I32, I32, I32, P, P, P, P, F32, P, P, P]),
    "lbm_step_f64": (I32, [P] * 12 + [I32] * 3 + [F64, F64, I32, F64, P]),
    "lbm_bc_f64": (I32, [P, P, P, I32, I32, I32, F64, P]),
    "lbm_update_uref_f64": (I32, [P] * 5 + [I32] * 3 + [P]),
    "lbm_build_flags": (I32, [ctypes.POINTER(Lattice), P, P, P, P]),
    "lbm_init_equilibrium": (I32, [ctypes.POINTER(Lattice), P, P]),
    "lbm_fused_step": (I32, [ctypes.POINTER(Lattice), P, P, U32, ctypes.POINTER(Tile), P]),
    "lbm_build_worklists": (I32, [ctypes.POINTER(Lattice), I32, P, P, P, P, P, P, P]),
    "lbm_build_worklists_noalloc": (I32, [ctypes.POINTER(Lattice), I32, P, P, P, P, P, P]),
    "lbm_init_equilibrium_h": (I32, [ctypes.POINTER(Lattice), P, ctypes.c_float, P]),
    "lbm_pack_populations": (I32, [ctypes.POINTER(Lattice), P, P, ctypes.c_float, P]),
    "lbm_unpack_populations": (I32, [ctypes.POINTER(Lattice), P, P, ctypes.c_float, P]),
    "lbm_fused_step_h": (I32, [ctypes.POINTER(Lattice), P, P, ctypes.c_float, ctypes.c_uint32,
                               ctypes.POINTER(Tile), P]),
    "lbm_profiles_scratch_doubles": (ctypes.c_longlong, [ctypes.POINTER(Lattice)]),
    "lbm_batch_pull_offsets_bytes": (I32, []),
    "lbm_batch_init": (I32, [ctypes.POINTER(Batch), P]),
    "lbm_batch_step_h": (I32, [ctypes.POINTER(Batch), I32, U32, ctypes.POINTER(Tile), P]),
    "lbm_gemm_bf16": (I32, [P, I32, P, I32, I32, I32, I32, P, I32, I32, P, P, P]),
    "lbm_lift_coarse": (I32, [ctypes.POINTER(Lattice), P, I32, I32, I32, I32, I32, F32, F32, P, P]),
    "lbm_nn_im2col": (I32, [P, I32, I32, I32, I32, P, P]),
    "lbm_nn_col2im": (I32, [P, I32, I32, I32, I32, P, P]),
    "lbm_nn_transpose": (I32, [P, ctypes.c_int64, I32, ctypes.c_int64, P, P]),
    "lbm_nn_act_grad": (I32, [P, P, ctypes.c_int64, I32, I32, P, P, P]),
    "lbm_nn_pool2": (I32, [P, I32, I32, I32, I32, P, P]),
    "lbm_nn_pool2_back": (I32, [P, I32, I32, I32, I32, P, I32, P]),
    "lbm_nn_up2_add": (I32, [P, P, I32, I32, I32, I32, P, P]),
    "lbm_nn_up2_back": (I32, [P, I32, I32, I32, I32, P, P]),
    "lbm_nn_mse": (I32, [P, I32, P, I32, P, ctypes.c_int64, F32, P, P, P]),
    "lbm_nn_adam": (I32, [P, P, P, P, ctypes.c_int64, F32, F32, F32, F32, I32, P, P]),
    "lbm_profiles": (I32, [ctypes.POINTER(Lattice), ctypes.c_double, P, P, P, P]),
    "lbm_body_forces_scratch_doubles": (ctypes.c_int64, [I32]),
    "lbm_batch_chunk_h": (I32, [ctypes.POINTER(Batch), I32, I32, ctypes.c_uint32, ctypes.c_uint32, P, P]),
    "lbm_body_forces": (I32, [ctypes.POINTER(Lattice), P, P, I32, ctypes.c_uint32, P, P, P]),
    "lbm_body_forces_h": (I32, [ctypes.POINTER(Lattice), P, F32, P, I32, ctypes.c_uint32, P, P, P]),
}
PROFILE_FIELDS = ("q", "uxx", "drho", "mass", "n_fluid", "top_n", "top_drho", "top_ux", "umax")

_lib = None
_lock = threading.Lock()


class LBMError(RuntimeError):
    pass


def load(require_build: bool = True) -> ctypes.CDLL:
    """Load the library (building it first when missing or older than its sources)."""
    global _lib
    with _lock:
        if _lib is None:
            if require_build and stale():
                build()
            if not os.path.exists(LIBPATH):
                raise LBMError(f"{LIBNAME} is not built and could not be built (nvcc missing?)")
            lib = ctypes.CDLL(LIBPATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(status: int, what: str) -> None:
    if status != LBM_OK:
        msg = load().lbm_last_error().decode(errors="replace")
        raise LBMError(f"{what} failed ({status}): {msg}")


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise LBMError("water_flow_simulation_b200 needs a CUDA device (B200, sm_100a); none is available")
    return torch
