"""The web viewer's case export (floodsim/web3d.py:28-86), with the 3D part on the GPU.

`export_case(run, label, c, res)` returns the reference's dictionary for one finished case:
the time-averaged velocity pooled over 2 x 2 horizontal blocks and quantised to int8
(base64), the pooled bed shear as uint16 centi-pascals, the bed height per y block, hulls,
propellers, the along-stream profiles and, with `c`, the comparison statistics.  The velocity
pooling and quantisation -- the only part that touches the whole lattice -- is
lbm_export_velocity on the device, reading the time-average sums where they are; only the
int8 blocks and the block speeds (for the 99.7th percentile) come back to the host.  The
rest works on (ny, nx) maps and is restated here from web3d.py:57-86.  The output equals
the reference's, key by key and byte by byte (tests/test_gpu_export.py against
tests/golden/export_*.npz, which the reference wrote).
"""
from __future__ import annotations

import base64
import ctypes

import numpy as np

from . import _native as nat
from .lbm3d import ctypes_ptr

STRIDE = 2


def _b64(a: np.ndarray) -> str:
    return base64.b64encode(np.ascontiguousarray(a).tobytes()).decode("ascii")


def velocity_int8(run):
    """(q int8 (nz, ny/2, nx/2, 3), scale, sp99): the int8 velocity blocks of
    floodsim/web3d.py:47-56 from the run's time averages (its current fields when nothing
    has been averaged yet, as Run3D.field(mean=True) falls back to them)."""
    import torch
    L, r = run.lbm, run.r
    lib = nat.load()
    lat = L._lattice()
    navg = int(run.navg)
    tmp = None
    if navg <= 0 or L._avg is None:
        tmp = torch.cat([L._ux, L._uy, L._uz])
        lat.avg = ctypes_ptr(tmp)
        navg = 1
    ref = ctypes.byref(lat)
    nb = int(lib.lbm_export_blocks(ref))
    if nb < 0:
        nat.check(nb, "lbm_export_blocks")
    dev = L.device
    pooled = torch.empty(4 * nb, dtype=torch.float32, device=dev)
    umax = torch.empty(1, dtype=torch.int32, device=dev)
    q = torch.empty(3 * nb, dtype=torch.int8, device=dev)
    sp = torch.empty(nb, dtype=torch.float32, device=dev)
    nat.check(lib.lbm_export_velocity(ref, navg, float(np.float32(r.vel)), ctypes_ptr(pooled), ctypes_ptr(umax),
                                      ctypes_ptr(q), ctypes_ptr(sp), L._stream()), "lbm_export_velocity")
    shape = (r.nz, r.ny // STRIDE, r.nx // STRIDE)
    qh = q.cpu().numpy().reshape(shape + (3,))
    sph = sp.cpu().numpy().reshape(shape)
    umax_f = float(np.array([umax.item()], np.int32).view(np.float32)[0]) or 1.0
    del tmp
    fluid = qh[..., 0] != -128
    return qh, umax_f / 126, float(np.percentile(sph[fluid], 99.7))


def export_case(run, label: str, c: dict | None, res: dict) -> dict:
    """floodsim/web3d.py:44-86 for one case after run_to_end; `res` = profiles(run)."""
    r = run.r
    q, scale, sp99 = velocity_int8(run)
    nz, ny2, nx2 = q.shape[:3]
    dxs = r.dx * STRIDE
    col = ~r.solid[:, :, 0]                     # bed height per y at the inlet (no hulls there)
    zb = np.where(col.any(0), col.argmax(0) * r.dx, r.h)
    zb2 = zb[:ny2 * STRIDE].reshape(ny2, STRIDE).min(1)
    tau = res["tau_bed"][:ny2 * STRIDE, :nx2 * STRIDE].reshape(ny2, STRIDE, nx2, STRIDE).max((1, 3))
    wet = tau > 0
    tau_top = float(max(np.percentile(tau[wet], 99.5) if wet.any() else 1.0, 1.0))
    tau_med = float(np.median(tau[wet])) if wet.any() else 1.0
    tq = np.clip(np.round(tau * 100), 0, 65535).astype(np.uint16)
    step = max(len(res["x"]) // 300, 1)
    out = dict(
        label=label, nx=int(nx2), ny=int(ny2), nz=int(nz), dxs=float(dxs), dz=float(r.dx),
        y0=float(r.y[0] - 0.5 * r.dx), L=float(nx2 * dxs), W=float(ny2 * dxs), h=float(r.h),
        V=float(r.V), Q=float(r.Q), S=float(r.S), scale=float(scale), u=_b64(q), sp99=float(sp99),
        tau=_b64(tq), tau_top=tau_top, tau_med=tau_med, zb=[round(float(v), 3) for v in zb2],
        hulls=[[round(float(v), 3) for v in hb] for hb in r.hulls],
        props=[dict(x=p["x"], y=p["y"], z=p["z"], D=p["D"], tilt=p["tilt"], yaw=p.get("yaw", 0.0)) for p in r.props],
        boat=r.fleet.boat.name if r.fleet.enabled else "",
        jet=bool(r.fleet.boat.is_jet) if r.fleet.enabled else False,
        prof=dict(x=[round(float(v), 2) for v in res["x"][::step]],
                  eta=[round(float(v) * 100, 3) for v in res["eta"][::step]],
                  umax=[round(float(v), 3) for v in res["umax"][::step]]),
    )
    if c:
        out["stats"] = {k: (None if (isinstance(v, float) and v != v) else round(float(v), 4))
                        for k, v in c.items() if isinstance(v, (int, float)) and not isinstance(v, bool)}
    return out
