"""CPU restatement of the tracer-particle step (test infrastructure only).

floodsim/reach3d.py:508-536 (Run3D.move_particles): each particle moves by the velocity of
the cell it is in (indices truncated and clipped), in m/s as float32 (lattice velocity x
vel), non-finite components set to 0, times dt in float32, added to its float64 position.  A
particle no longer finite, out of the domain (x index past nx-2, y or z out of range) or in
a solid cell is restarted at the inlet from a random generator; this restatement returns the
moved positions and the mask of restarted particles, whose positions it leaves as moved.
tests/golden/particles_*.npz, written by the reference itself, pin it: the positions of the
particles not restarted bit for bit, and the restart count.  Only tests import this module.
"""
from __future__ import annotations

import numpy as np


def move(P, ux, uy, uz, solid, vel, dt, dx):
    """(P moved (n, 3) float64, restarted mask (n,)) for flat float32 lattice-unit velocity
    fields in the reference layout."""
    nz, ny, nx = solid.shape
    P = np.array(P, np.float64)
    ix = np.clip((P[:, 0] / dx).astype(int), 0, nx - 1)
    iy = np.clip((P[:, 1] / dx).astype(int), 0, ny - 1)
    iz = np.clip((P[:, 2] / dx).astype(int), 0, nz - 1)
    cell = ix + nx * (iy + ny * iz)
    u = np.stack([ux[cell], uy[cell], uz[cell]], 1) * vel
    with np.errstate(over="ignore", invalid="ignore"):
        P += np.nan_to_num(u, nan=0.0, posinf=0.0, neginf=0.0) * dt
    fin = np.isfinite(P).all(1)
    Q = np.where(fin[:, None], P, -1.0)
    jx, jy, jz = ((Q[:, k] / dx).astype(int) for k in range(3))
    out = ~fin | (jx < 0) | (jx >= nx - 1) | (jy < 0) | (jy >= ny) | (jz < 0) | (jz >= nz)
    bad = out.copy()
    ok = ~out
    bad[ok] = solid[jz[ok], jy[ok], jx[ok]]
    return P, bad
