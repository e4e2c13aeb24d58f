"""CPU oracle for the D3Q19 hot path (test infrastructure only).

This module is the checker that the CUDA path is compared against. Only the test
suite, the smoke check and the CPU-baseline leg of ``bench.py`` import it; the
product package never does, and it has no fallback role.

It wraps ``lbm_oracle.c`` (a C restatement of the reference's Numba twin,
``floodsim/lbm3d.py:179-330``) through ctypes, and restates in NumPy the two
host-side pieces of ``LBM3D`` that feed the kernels:

* ``equilibrium_init`` -- the 1D-profile start ``f = feq(rho=1, u=(uin,0,0))``
  broadcast along x, solids at rest (``floodsim/lbm3d.py:362-364, 377-384``);
* ``wall_mask`` -- the per-cell 19-bit set of directions whose pull source is a
  wall (``floodsim/lbm3d.py:50-58``), used for the bit-exact flag-map checks.

``OracleLBM`` drives the C functions with the same array set and ``step(n)``
contract as ``LBM3D`` (``floodsim/lbm3d.py:342-412``), in FP32 (Numba typing) or
FP64.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "lbm_oracle.c")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liblbm_oracle.so")

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
MIRZ = np.array([0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16])


def build_oracle(force: bool = False) -> str:
    """Compile lbm_oracle.c into oracle/_build (gcc, OpenMP, no FP contraction)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    tmp = LIB + f".tmp{os.getpid()}"
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
                           "-fno-fast-math", "-Wall", "-o", tmp, SRC, "-lm"])
    os.replace(tmp, LIB)
    return LIB


def build_oracle_timing(out_dir: str) -> str:
    """Compile lbm_oracle.c for timing only, into out_dir: -O3 for this host's CPU with
    -ffast-math, the compile mode the reference asks Numba for (fastmath=True,
    floodsim/lbm3d.py:186).  Same source and algorithm; the rounding is no longer the
    Numba path's bit for bit, so only the CPU baseline of bench.py uses it, never a parity
    test (tests/test_oracle_timing.py checks that it stays within the parity bar)."""
    os.makedirs(out_dir, exist_ok=True)
    out = os.path.join(out_dir, "liblbm_oracle_timing.so")
    tmp = out + f".tmp{os.getpid()}"
    subprocess.check_call(["gcc", "-O3", "-march=native", "-ffast-math", "-fopenmp", "-fPIC", "-shared",
                           "-o", tmp, SRC, "-lm"])
    os.replace(tmp, out)
    return out


_lib = None
_timing_libs = {}


def _declare(L: ctypes.CDLL) -> ctypes.CDLL:
    P, I64 = ctypes.c_void_p, ctypes.c_int64
    L.oracle_step_f32.argtypes = [P] * 12 + [I64] * 3 + [ctypes.c_float] * 2
    L.oracle_step_f64.argtypes = [P] * 12 + [I64] * 3 + [ctypes.c_double] * 2
    L.oracle_step_f32_x.argtypes = [P] * 12 + [I64] * 3 + [P, ctypes.c_float]
    L.oracle_step_f64_x.argtypes = [P] * 12 + [I64] * 3 + [P, ctypes.c_double]
    L.oracle_bc_f32.argtypes = [P] * 3 + [I64] * 3 + [ctypes.c_float]
    L.oracle_bc_f64.argtypes = [P] * 3 + [I64] * 3 + [ctypes.c_double]
    L.oracle_update_uref_f32.argtypes = [P] * 5 + [I64] * 3
    L.oracle_update_uref_f64.argtypes = [P] * 5 + [I64] * 3
    L.oracle_num_threads.restype = ctypes.c_int
    L.oracle_body_forces_f32.argtypes = [P] * 3 + [ctypes.c_int] + [P] * 6 + [I64] * 3 + [P]
    return L


def timing_lib(out_dir: str) -> ctypes.CDLL:
    """The timing build (build_oracle_timing) loaded through ctypes, built once per out_dir."""
    if out_dir not in _timing_libs:
        _timing_libs[out_dir] = _declare(ctypes.CDLL(build_oracle_timing(out_dir)))
    return _timing_libs[out_dir]


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = _declare(ctypes.CDLL(build_oracle()))
    return _lib


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data


def equilibrium_init(solid: np.ndarray, uin: np.ndarray, dtype=np.float32) -> np.ndarray:
    """Initial populations, floodsim/lbm3d.py:362-364 and 377-384.

    The arithmetic keeps NumPy's own promotion rules (float64 W and c_i terms,
    a float32 ``1.5*u*u`` product), so the float32 result is bit-identical to
    the reference's start state.
    """
    nz, ny, nx = solid.shape
    n = solid.size
    u0 = np.broadcast_to(uin[:, :, None], solid.shape).copy()
    u0[solid] = 0
    ux = u0.ravel().astype(dtype)
    r = np.ones(solid.shape, dtype).ravel()
    f = np.empty(19 * n, dtype)
    for i in range(19):
        cu = 3 * CX[i] * ux
        f[i * n:(i + 1) * n] = W[i] * r * (1 + cu + 0.5 * cu * cu - 1.5 * ux * ux)
    return f


def wall_mask(solid: np.ndarray) -> np.ndarray:
    """uint32 (nz,ny,nx): bit i set when direction i's pull source is a wall.

    floodsim/lbm3d.py:50-58: x-out-of-range directions are plain copies (never
    walls); a source above the lid is mirrored into the same layer; a source
    outside the y range, below the bed (z<0) or on a solid cell is a wall.
    Solid cells themselves get mask 0.
    """
    nz, ny, nx = solid.shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    m = np.zeros(solid.shape, np.uint32)
    for i in range(1, 19):
        xs, ys, zs = x - CX[i], y - CY[i], z - CZ[i]
        xin = (xs >= 0) & (xs < nx)
        zs = np.where(zs >= nz, z, zs)
        oob = (ys < 0) | (ys >= ny) | (zs < 0)
        sol = solid[np.clip(zs, 0, nz - 1), np.clip(ys, 0, ny - 1), np.clip(xs, 0, nx - 1)]
        wall = xin & (oob | sol)
        m |= wall.astype(np.uint32) << np.uint32(i)
    m[solid] = 0
    return m


class OracleLBM:
    """The reference solver state and step loop on the CPU (floodsim/lbm3d.py:333-412)."""

    def __init__(self, solid, Fx, Fy, Fz, uin, tau0, cs=0.17, cf_wall=None, precision="f32", sponge=None,
                 clib=None):
        """clib: the C library to step with (default: the exact build, lib())."""
        self._clib = clib
        dt = np.float32 if precision == "f32" else np.float64
        self.dt, self.precision = dt, precision
        self.nz, self.ny, self.nx = solid.shape
        self.N = solid.size
        self.tau0, self.csmag2 = float(tau0), float(cs * cs)
        self.tau0_x = None
        if sponge is not None and sponge[0] > 0:
            # optional outlet sponge (not in the reference): tau0 + (tau_s - tau0) s^2 over the
            # last K columns, s = (x - (nx - K) + 1) / K, in the storage precision
            K, ts = int(sponge[0]), sponge[1]
            x = np.arange(self.nx)
            s_ = (np.maximum(x - (self.nx - K) + 1, 0).astype(dt)) / dt(K)
            t0 = dt(self.tau0)
            tx = t0 + (dt(ts) - t0) * (s_ * s_)
            self.tau0_x = np.ascontiguousarray(np.where(x >= self.nx - K, tx, t0).astype(dt))
        A = lambda a: np.ascontiguousarray(np.asarray(a).ravel(), dtype=dt)  # noqa: E731
        self.solid = np.ascontiguousarray(solid.astype(np.uint8).ravel())
        self.Fx, self.Fy, self.Fz = A(Fx), A(Fy), A(Fz)
        self.uin = A(uin)
        self.rho = np.ones(self.N, dt)
        self.ux = np.zeros(self.N, dt)
        self.uy = np.zeros(self.N, dt)
        self.uz = np.zeros(self.N, dt)
        self.cfw = A(cf_wall if cf_wall is not None else np.zeros(solid.shape, np.float32))
        self.uref = np.zeros(self.N, dt)
        uin32 = np.asarray(uin, np.float32)
        self.f = equilibrium_init(solid, uin32 if dt is np.float32 else np.asarray(uin, np.float64), dt)
        self.f2 = self.f.copy()
        self.nstep = 0

    def step(self, n: int = 1) -> None:
        L = self._clib or lib()
        nx, ny, nz = self.nx, self.ny, self.nz
        f32 = self.dt is np.float32
        if self.tau0_x is None:
            st, t0 = (L.oracle_step_f32 if f32 else L.oracle_step_f64), self.tau0
        else:
            st, t0 = (L.oracle_step_f32_x if f32 else L.oracle_step_f64_x), _p(self.tau0_x)
        bc = L.oracle_bc_f32 if f32 else L.oracle_bc_f64
        for _ in range(n):
            st(_p(self.f), _p(self.f2), _p(self.solid), _p(self.Fx), _p(self.Fy), _p(self.Fz),
               _p(self.rho), _p(self.ux), _p(self.uy), _p(self.uz), _p(self.cfw), _p(self.uref),
               nx, ny, nz, t0, self.csmag2)
            bc(_p(self.f2), _p(self.solid), _p(self.uin), nx, ny, nz, 1.0)
            self.f, self.f2 = self.f2, self.f
        self.nstep += n

    def update_uref(self, bedwall: np.ndarray) -> None:
        """Column-mean wall-model speed (floodsim/reach3d.py:412-418)."""
        L = self._clib or lib()
        bw = np.ascontiguousarray(np.asarray(bedwall).astype(np.uint8).ravel())
        fn = L.oracle_update_uref_f32 if self.dt is np.float32 else L.oracle_update_uref_f64
        fn(_p(self.ux), _p(self.uy), _p(self.solid), _p(bw), _p(self.uref), self.nx, self.ny, self.nz)

    def run_chunks(self, nsteps: int, bedwall=None, every: int = 20) -> None:
        """Steps in chunks of `every`, refreshing uref before each chunk, as
        Run3D.advance does (floodsim/reach3d.py:424-442)."""
        k = 0
        while k < nsteps:
            m = min(every, nsteps - k)
            if bedwall is not None:
                self.update_uref(bedwall)
            self.step(m)
            k += m

    def shape3(self, a):
        return a.reshape(self.nz, self.ny, self.nx)


class OracleRun3D:
    """Run3D's time loop on the oracle (floodsim/reach3d.py:378-453): the smoothstep force
    ramp F0 * f^2 (3 - 2f) over t_ramp (reach3d.py:401, 431-437, applied by rewriting the
    float32 force arrays at the start of every chunk), the column-mean uref refresh before
    every chunk (reach3d.py:438-439), and the float32 time-average sums added after every
    chunk that ends at t >= t_avg (reach3d.py:443-451).  Chunks of at most 20 steps."""

    AVG_KEYS = ("ux", "uy", "uz", "rho", "sp", "uxx")

    def __init__(self, solid, Fx, Fy, Fz, uin, tau0, cs, cf_wall, bedwall, dt, t_ramp, t_avg):
        self.lbm = OracleLBM(solid, Fx, Fy, Fz, uin, tau0, cs, cf_wall)
        self.bedwall = bedwall
        self.dt, self.t_ramp, self.t_avg = dt, t_ramp, t_avg
        self.t = 0.0
        self.F0 = (self.lbm.Fx.copy(), self.lbm.Fy.copy(), self.lbm.Fz.copy())
        self.ramp_done = t_ramp <= 0
        if not self.ramp_done:
            for a in (self.lbm.Fx, self.lbm.Fy, self.lbm.Fz):
                a *= 0
        self.sum = {k: np.zeros(self.lbm.N, np.float32) for k in self.AVG_KEYS}
        self.navg = 0

    def advance(self, nsteps: int) -> None:
        L = self.lbm
        k = 0
        while k < nsteps:
            m = min(20, nsteps - k)
            if not self.ramp_done:
                f = min(self.t / self.t_ramp, 1.0)
                f = np.float32(f * f * (3 - 2 * f))
                L.Fx = np.ascontiguousarray(self.F0[0] * f)
                L.Fy = np.ascontiguousarray(self.F0[1] * f)
                L.Fz = np.ascontiguousarray(self.F0[2] * f)
                self.ramp_done = f >= 1.0
            if self.bedwall is not None:
                L.update_uref(self.bedwall)
            L.step(m)
            k += m
            self.t += m * self.dt
            if self.t >= self.t_avg:
                s = self.sum
                s["ux"] += L.ux
                s["uy"] += L.uy
                s["uz"] += L.uz
                s["rho"] += L.rho
                s["sp"] += np.sqrt(L.ux * L.ux + L.uy * L.uy + L.uz * L.uz)
                s["uxx"] += L.ux * L.ux
                self.navg += 1


def body_forces(o: "OracleLBM", body: np.ndarray, nbody: int) -> np.ndarray:
    """Momentum-exchange force on each body (hull) for the next step's bounce-back, from the
    oracle's state (oracle_body_forces_f32): (nbody, 3) float64, lattice units."""
    b = np.ascontiguousarray(np.asarray(body, np.uint8).ravel())
    out = np.zeros(3 * nbody, np.float64)
    (o._clib or lib()).oracle_body_forces_f32(_p(o.f), _p(o.solid), _p(b), nbody, _p(o.rho), _p(o.ux), _p(o.uy),
                                              _p(o.uz), _p(o.cfw), _p(o.uref), o.nx, o.ny, o.nz, _p(out))
    return out.reshape(nbody, 3)

