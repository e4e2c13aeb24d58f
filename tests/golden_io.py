"""Readers for the golden fixtures written by tests/golden/make_golden.py."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STEP_CASES = ("mini_cfg1", "mini_tug", "mini_jet", "mini_nowm")
REACH_CASES = ("cfg1", "tug_trap", "jet_flood", "curtain_nowm", "shallow_outboard", "base_rect")
STEP_NS = (1, 2, 5, 25)


class Case:
    """One fixture: the reference's build_reach outputs (and, for steps_*, its solver states)."""

    def __init__(self, path):
        self.path = path
        d = np.load(path)
        self.d = d
        self.spec = json.loads(str(d["spec"]))
        self.meta = json.loads(str(d["meta"]))
        self.nx, self.ny, self.nz = (int(v) for v in d["dims"])
        self.shape = (self.nz, self.ny, self.nx)
        N = self.N = self.nx * self.ny * self.nz
        (self.dx, self.dt, self.V, self.A, self.W, self.h, self.Q, self.S,
         self.tau0, self.cs) = (float(v) for v in d["scalars"])
        self.solid = np.unpackbits(d["solid"])[:N].astype(bool).reshape(self.shape)
        self.F = []
        for nm in ("Fx", "Fy", "Fz"):
            a = np.zeros(N, np.float32)
            a[d[nm + "_idx"]] = d[nm + "_val"]
            self.F.append(a.reshape(self.shape))
        self.cf = self.bedwall = None
        if "cf_idx" in d:
            cf = np.zeros(N, np.float32)
            cf[d["cf_idx"]] = d["cf_val"]
            self.cf = cf.reshape(self.shape)
            self.bedwall = np.unpackbits(d["bedwall"])[:N].astype(bool).reshape(self.shape)
        self.uin_lb = d["uin_lb"]
        self.uin_phys = d["uin_phys"]
        self.y, self.zc = d["y"], d["zc"]

    def state(self, n):
        return {k: self.d[f"{k}_{n}"] for k in ("rho", "ux", "uy", "uz")}


def load_step_case(name) -> Case:
    return Case(os.path.join(GOLDEN, f"steps_{name}.npz"))


def load_reach_case(name) -> Case:
    return Case(os.path.join(GOLDEN, f"reach_{name}.npz"))


ADVANCE_CASES = ("mini_tug", "mini_cfg1")


def load_advance_case(name) -> Case:
    """advance_<name>.npz: the reference's Run3D.advance in short chunks with the force ramp and
    the averaging active (fields, uref and sums after chunk k under keys *_c<k>)."""
    return Case(os.path.join(GOLDEN, f"advance_{name}.npz"))
