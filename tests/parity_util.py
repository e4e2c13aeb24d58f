"""Shared helpers for the parity tests: the oracle on a golden case and its own sensitivity.

The reference's update is chaotic near walls (the wall function normalises a
tangential velocity that can be tiny), so after a few steps any change of
rounding grows.  ``oracle_spread`` measures that growth for the reference path
itself: the oracle is run twice, once from a start state perturbed by one float32
ulp per population, and the max-norm difference of the velocity fields
(relative to max|u|) is recorded after every step.  A CUDA result that differs
from the oracle by no more than this spread differs by no more than the
reference's own rounding does.
"""
from __future__ import annotations

import functools

import numpy as np

from oracle.oracle import OracleLBM


def case_arrays(c, crop=None):
    solid, F, cf, bw = c.solid, list(c.F), c.cf, c.bedwall
    if crop is not None:
        solid = solid[..., :crop]
        F = [a[..., :crop] for a in F]
        cf = None if cf is None else cf[..., :crop]
        bw = None if bw is None else bw[..., :crop]
    return solid, F, cf, bw


def make_oracle(c, crop=None, precision="f32"):
    solid, F, cf, _ = case_arrays(c, crop)
    o = OracleLBM(solid, *F, c.uin_lb, c.tau0, c.cs, cf, precision=precision)
    if "csmag2" in c.d:
        o.csmag2 = float(c.d["csmag2"])
    return o


def rel_u_error(a, b):
    """max over ux,uy,uz of max|a-b| / max|b| (a, b: objects or dicts of host arrays)."""
    get = lambda o, k: o[k] if isinstance(o, dict) else getattr(o, k)  # noqa: E731
    umax = max(float(np.abs(get(b, k)).max()) for k in ("ux", "uy", "uz"))
    return max(float(np.abs(np.asarray(get(a, k)) - get(b, k)).max()) for k in ("ux", "uy", "uz")) / umax


@functools.lru_cache(maxsize=None)
def _spread(path, crop, nsteps):
    from golden_io import Case
    c = Case(path)
    _, _, _, bw = case_arrays(c, crop)
    a, b = make_oracle(c, crop), make_oracle(c, crop)
    sgn = np.random.default_rng(1).choice([-1.0, 1.0], b.f.size).astype(np.float32)
    b.f = np.nextafter(b.f, b.f + sgn).astype(np.float32)
    out = []
    for _ in range(nsteps):
        for o in (a, b):
            if bw is not None:
                o.update_uref(bw)
            o.step(1)
        out.append(rel_u_error(b, a))
    return tuple(out)


def oracle_spread(c, nsteps, crop=None):
    """Per-step 1-ulp sensitivity of the reference path on case `c` (tuple, index n-1 = after n steps)."""
    return _spread(c.path, crop, nsteps)


def bound(c, n, tol, crop=None, factor=2.0):
    """The parity bar after n steps: tol, or `factor` x the reference's own 1-ulp spread if larger."""
    return max(tol, factor * oracle_spread(c, max(n, 1), crop)[n - 1])


_SPREADS = {}


def case_spread(key, c, nsteps, crop=None):
    """oracle_spread for a case built in the test (not a golden file), cached under `key`."""
    k = (key, crop, nsteps)
    if k not in _SPREADS:
        _, _, _, bw = case_arrays(c, crop)
        a, b = make_oracle(c, crop), make_oracle(c, crop)
        sgn = np.random.default_rng(1).choice([-1.0, 1.0], b.f.size).astype(np.float32)
        b.f = np.nextafter(b.f, b.f + sgn).astype(np.float32)
        out = []
        for _ in range(nsteps):
            for o in (a, b):
                if bw is not None:
                    o.update_uref(bw)
                o.step(1)
            out.append(rel_u_error(b, a))
        _SPREADS[k] = tuple(out)
    return _SPREADS[k]


def case_bound(key, c, n, tol, crop=None, factor=2.0):
    """bound() for a case built in the test."""
    return max(tol, factor * case_spread(key, c, max(n, 1), crop)[n - 1])
