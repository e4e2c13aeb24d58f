"""The reach builder with its three-dimensional arrays made on the GPU.

`build_reach_device(sec, h, Q, S, fleet, cfg, bed_bumps=None)` returns the same Reach as
`reach3d.build_reach` (floodsim/reach3d.py:201-297, wall_cf 315-343) -- same scalars, inlet
profile, hulls, propellers and notes -- with solid, Fx, Fy, Fz, cf and bedwall as torch
tensors on the GPU, bit for bit equal to the host builder's arrays.  At 259.6M cells the
host builder spends most of its ~18 s and ~6 GB on those full-size NumPy arrays, and the
solver then copies ~5 GB of them to the device; here the host computes only what is one-
or two-dimensional or sparse, and two kernels (lbm_build_reach_masks, lbm_build_reach_walls)
write the full arrays where the solver reads them:

* the bed as a per-column count of cell centres below the bed level (kb) and the columns
  outside the top width;
* the hulls as y ranges per x column above a keel index, recorded by running the host's own
  boat placement (`reach3d._place_fleet`) on a stand-in solid that answers reads from kb,
  the outside columns and the hulls carved so far;
* the propeller and jet forces as the sparse cells of their disks, accumulated by the same
  placement code into a sparse stand-in, in the same float32 order, then scattered on the
  device and scaled to lattice units there.

A Reach built here feeds Run3D, BatchRun and profiles_device directly; `to_host(reach)`
gives the NumPy version for host-side helpers.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from . import _native as nat
from .reach3d import (RHO, G, Reach, _inlet_profile, _place_fleet, _time_step, bed_level, lattice_grid, log_cf)


class _ColumnSolid:
    """Stand-in for the (nz, ny, nx) solid array during boat placement: reads of index boxes
    are computed from the bed columns and the hull carves so far; writes (hull carving) are
    recorded as (x, y0, y1, z0) segments."""

    def __init__(self, kb, outside, nz):
        self.kb, self.outside, self.nz = kb, outside, nz
        self.segs = []

    def __setitem__(self, key, value):
        iz, iy, ix = (np.asarray(k).ravel() for k in key)
        if not (value is True or np.all(value)):
            raise ValueError("only hull carving (True) is recorded")
        if iz.size == 0 or iy.size == 0:
            return
        if not (np.array_equal(iy, np.arange(iy[0], iy[-1] + 1)) and iz[-1] == self.nz - 1
                and np.array_equal(iz, np.arange(iz[0], self.nz))):
            raise ValueError("a hull carve must be one y range above a keel index")
        for x in ix:
            self.segs.append((int(x), int(iy[0]), int(iy[-1]), int(iz[0])))

    def __getitem__(self, key):
        iz, iy, ix = (np.asarray(k).ravel() for k in key)
        out = (iz[:, None, None] < self.kb[np.ix_(iy, ix)][None]) | self.outside[iy][None, :, None]
        for x, y0, y1, z0 in self.segs:
            kx = np.flatnonzero(ix == x)
            if kx.size:
                sel = np.ix_(iz >= z0, (iy >= y0) & (iy <= y1), kx)
                out[sel] = True
        return out


class _SparseField:
    """Stand-in for a float32 (nz, ny, nx) force array: `F[box] += v` on index boxes, kept as
    sorted flat indices and float32 values."""

    def __init__(self, shape):
        self.nz, self.ny, self.nx = shape
        self.keys = np.zeros(0, np.int64)
        self.vals = np.zeros(0, np.float32)

    def _flat(self, key):
        iz, iy, ix = (np.asarray(k).ravel().astype(np.int64) for k in key)
        return (ix[None, None, :] + self.nx * (iy[None, :, None] + self.ny * iz[:, None, None]))

    def __getitem__(self, key):
        f = self._flat(key)
        pos = np.searchsorted(self.keys, f)
        pos_c = np.minimum(pos, max(len(self.keys) - 1, 0))
        hit = (pos < len(self.keys)) & (self.keys[pos_c] == f) if len(self.keys) else np.zeros(f.shape, bool)
        out = np.zeros(f.shape, np.float32)
        out[hit] = self.vals[pos_c[hit]]
        return out

    def __setitem__(self, key, value):
        f = self._flat(key).ravel()
        v = np.broadcast_to(np.asarray(value, np.float32), self._flat(key).shape).ravel()
        keys = np.concatenate([self.keys, f])
        vals = np.concatenate([self.vals, v])
        order = np.argsort(keys, kind="stable")
        keys, vals = keys[order], vals[order]
        last = np.ones(len(keys), bool)                  # for repeated cells the new value wins
        last[:-1] = keys[1:] != keys[:-1]
        self.keys, self.vals = keys[last], vals[last]


def _columns(sec, h, cfg, bed_bumps):
    """Grid and bed of build_reach (floodsim/reach3d.py:204-217) without 3D arrays."""
    fp, Wtop, dx, nx, ny, nz = lattice_grid(sec, h, cfg)
    y = (np.arange(ny) - ny / 2 + 0.5) * dx
    zc = (np.arange(nz) + 0.5) * dx
    zb = bed_level(y, sec)
    outside = np.abs(y) > Wtop / 2
    if bed_bumps is None:
        kb = np.broadcast_to(np.searchsorted(zc, zb, side="left")[:, None], (ny, nx))
    else:
        zb3 = zb[:, None] + bed_bumps((np.arange(nx) + 0.5) * dx, y)
        kb = np.searchsorted(zc, zb3.ravel(), side="left").reshape(ny, nx)
    kb = np.ascontiguousarray(kb, np.int32)
    return fp, Wtop, dx, nx, ny, nz, y, zc, outside, kb


class Plan:
    """What the host computes for a device build: scalars, inlet profile, boats, the bed as
    columns (kb, outside), the hull segments and the sparse forces (N/m^3, float32)."""


def plan_reach(sec, h, Q, S, fleet, cfg, bed_bumps=None) -> Plan:
    """The host part of build_reach_device (no array larger than a cross-section or a
    propeller's disk box)."""
    P = Plan()
    notes = []
    fp, Wtop, dx, nx, ny, nz, y, zc, outside, kb = _columns(sec, h, cfg, bed_bumps)
    if fp > 0 and sec.Bf > fp:
        notes.append(f"floodplain modelled to {fp:g} m per side (the domain edge is a wall)")
    sol2 = (np.arange(nz)[:, None] < kb[:, 0][None, :]) | outside[None, :]
    fluid2 = ~sol2
    prof = _inlet_profile(fluid2, dx, cfg.wall_model)
    A = fluid2.sum() * dx * dx
    V = Q / A
    uin = prof * (V * fluid2.sum() / prof.sum())
    solid_h = _ColumnSolid(kb, outside, nz)
    F = [_SparseField((nz, ny, nx)) for _ in range(3)]
    hulls, props = [], []
    Xc = (np.arange(nx) + 0.5) * dx
    if fleet.enabled and fleet.n_boats > 0:
        hulls, props = _place_fleet(fleet, sec, h, cfg, solid_h, *F, Xc, y, zc, dx, notes)
        notes = list(dict.fromkeys(notes))
    keys = F[0].keys
    for f in F[1:]:
        if not np.array_equal(f.keys, keys):
            raise RuntimeError("force components cover different cells")
    fx, fy, fz = (f.vals for f in F)
    fmax = float(np.sqrt(fx ** 2 + fy ** 2 + fz ** 2).max()) if len(keys) else 0.0
    dt = _time_step(cfg, dx, nx, V, uin, props, None, None, None, fmax=fmax)
    segs = sorted(solid_h.segs)
    seg_off = np.zeros(nx + 1, np.int64)
    np.add.at(seg_off, np.array([sg[0] + 1 for sg in segs], np.int64), 1)
    kb_eff = np.where(outside[:, None], nz, kb)
    hcol = np.maximum((nz - kb_eff) * dx, dx)
    P.__dict__.update(
        sec=sec, cfg=cfg, fleet=fleet, h=h, Q=Q, S=S, dx=dx, dt=dt, nx=nx, ny=ny, nz=nz, y=y, zc=zc, W=Wtop, A=A,
        V=V, uin=uin, hulls=hulls, props=props, notes=notes, kb=kb, outside=outside,
        seg_off=np.cumsum(seg_off).astype(np.int32),
        segs=np.array([sg[1:] for sg in segs], np.int32).reshape(-1, 3) if segs else np.zeros((1, 3), np.int32),
        keys=keys, F=(fx, fy, fz), k=dt * dt / (RHO * dx),
        cf_col=(G * sec.n * sec.n / hcol ** (1 / 3)).astype(np.float32),
        cf_hull=np.float32(log_cf(0.5 * dx, cfg.hull_ks)))
    return P


def build_reach_device(sec, h, Q, S, fleet, cfg, bed_bumps=None, device=None) -> Reach:
    """reach3d.build_reach with the full arrays built on the GPU (torch tensors)."""
    import torch
    nat.require_cuda()
    lib = nat.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    P = plan_reach(sec, h, Q, S, fleet, cfg, bed_bumps)
    nx, ny, nz = P.nx, P.ny, P.nz
    N = nx * ny * nz
    st = torch.cuda.current_stream(dev).cuda_stream
    T = lambda a, dt_: torch.as_tensor(np.ascontiguousarray(a, dt_), device=dev)  # noqa: E731
    p = lambda a: a.data_ptr()  # noqa: E731
    kb_d, out_d = T(P.kb, np.int32), T(P.outside, np.uint8)
    off_d, seg_d = T(P.seg_off, np.int32), T(P.segs, np.int32)
    solid = torch.empty(N, dtype=torch.uint8, device=dev)
    bed = torch.empty(N, dtype=torch.uint8, device=dev)
    nat.check(lib.lbm_build_reach_masks(nx, ny, nz, p(kb_d), p(out_d), p(off_d), p(seg_d), p(solid), p(bed), st),
              "lbm_build_reach_masks")
    kf = torch.tensor(np.float32(P.k), device=dev)
    Fd = []
    for vals in P.F:
        a = torch.zeros(N, dtype=torch.float32, device=dev)
        if len(P.keys):
            a[T(P.keys, np.int64)] = T(vals, np.float32)
        Fd.append((a * kf).view(nz, ny, nx))
    cf = bedwall = None
    if P.cfg.wall_model:
        cf_d = torch.empty(N, dtype=torch.float32, device=dev)
        bw_d = torch.empty(N, dtype=torch.uint8, device=dev)
        scratch = torch.empty(N, dtype=torch.uint8, device=dev)
        cf_col = T(np.array(np.broadcast_to(P.cf_col if P.cf_col.ndim == 2 else P.cf_col[:, None], (ny, nx)),
                            np.float32), np.float32)
        nat.check(lib.lbm_build_reach_walls(nx, ny, nz, p(solid), p(bed), p(scratch), p(cf_col), float(P.cf_hull),
                                            p(cf_d), p(bw_d), st), "lbm_build_reach_walls")
        del scratch
        cf, bedwall = cf_d.view(nz, ny, nx), bw_d.view(nz, ny, nx).bool()
    del bed
    return Reach(sec=sec, cfg=cfg, fleet=fleet, h=h, Q=Q, S=S, dx=P.dx, dt=P.dt, nx=nx, ny=ny, nz=nz, y=P.y,
                 zc=P.zc, solid=solid.view(nz, ny, nx).bool(), uin_phys=P.uin, Fx=Fd[0], Fy=Fd[1], Fz=Fd[2], cf=cf,
                 bedwall=bedwall, hulls=P.hulls, props=P.props, notes=P.notes, W=P.W, A=P.A, V=P.V)


def to_host(reach: Reach) -> Reach:
    """The same Reach with NumPy arrays (for the host-side helpers)."""
    def h(a):
        return a if a is None or isinstance(a, np.ndarray) else a.cpu().numpy()
    return replace(reach, solid=h(reach.solid), Fx=h(reach.Fx), Fy=h(reach.Fy), Fz=h(reach.Fz), cf=h(reach.cf),
                   bedwall=h(reach.bedwall))
