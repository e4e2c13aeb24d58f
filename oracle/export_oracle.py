"""CPU restatement of the web viewer's velocity export (test infrastructure only).

floodsim/web3d.py:35-56 (`_pool` and the int8 part of `export_case`): the time-averaged
velocity, in m/s, is averaged over the fluid cells of each 2 x 2 horizontal block, then
quantised to int8 with one scale for the case (the largest |component| / 126), round half to
even, clipped to +-126, and -128 marks a block without fluid.  The arithmetic keeps NumPy's
float32 promotion of the reference (mean = sum / navg and x vel in float32; block sums in the
order NumPy's two-axis reduction adds them); tests/golden/export_*.npz, written by the
reference itself, pin it bit for bit.  Only tests import this module.
"""
from __future__ import annotations

import numpy as np

STRIDE = 2


def mean_field(sum_flat, navg, vel, shape):
    """Run3D.field(name, mean=True) for a velocity component (floodsim/reach3d.py:474-486)."""
    a = np.asarray(sum_flat, np.float32) / np.float32(navg)
    return a.reshape(shape) * np.float32(vel)


def pool(a, fl, s=STRIDE):
    """floodsim/web3d.py:35-41: the fluid-cell mean of each s x s horizontal block."""
    nz, ny, nx = a.shape
    ny2, nx2 = ny // s, nx // s
    blocks = (a * fl)[:, :ny2 * s, :nx2 * s].reshape(nz, ny2, s, nx2, s)
    n = fl[:, :ny2 * s, :nx2 * s].reshape(nz, ny2, s, nx2, s).sum((2, 4))
    tot = blocks.sum(4).sum(2)                 # each row's pair first, then the rows
    return np.where(n > 0, tot / np.maximum(n, np.float32(1)), np.float32(0)).astype(np.float32), n > 0


def velocity_int8(sums, navg, vel, solid, s=STRIDE):
    """(q int8 (nz, ny/s, nx/s, 3), scale, sp99) of floodsim/web3d.py:47-56 from the float32
    time-average sums of ux, uy, uz (flat, reference layout)."""
    fl = (~solid).astype(np.float32)
    comps, fluid = [], None
    for k in range(3):
        a, fluid = pool(mean_field(sums[k], navg, vel, solid.shape), fl, s)
        comps.append(a)
    umax = max(float(np.abs(a).max()) for a in comps) or 1.0
    scale = umax / 126
    q = np.stack([np.clip(np.round(a / np.float32(scale)), -126, 126) for a in comps], -1).astype(np.int8)
    q[~fluid] = -128
    sp = np.sqrt(comps[0] * comps[0] + comps[1] * comps[1] + comps[2] * comps[2])
    sp99 = float(np.percentile(sp[fluid], 99.7))
    return q, scale, sp99
