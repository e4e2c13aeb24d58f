"""Float64 runs of a boat case on the GPU, the reference of the accuracy statements.

The reference algorithm (floodsim/lbm3d.py:31-175) with float64 populations, fields and
arithmetic, stepped with Run3D.advance's cadence (floodsim/reach3d.py:424-453): 20-step
chunks, the smoothstep force ramp applied to the float32 forces, the column-mean wall speed
refreshed before each chunk, and the time averages of rho, u, |u| and ux^2 at the chunk ends
inside the averaging window.  The kernels are lbm_step_f64 / lbm_bc_f64 /
lbm_update_uref_f64 of the library; they agree with the CPU float64 oracle to rounding
(tests/test_gpu_fp64.py), and reach sizes (36M cells x 20k steps) the CPU oracle cannot.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat
from .reach3d import Run3D

W64 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float64)
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0], np.float64)


class Solver64:
    """One boat case (a Reach) in float64 on the GPU."""

    def __init__(self, reach, device=None, sponge=None):
        import torch
        nat.require_cuda()
        self.torch, self.lib = torch, nat.load()
        self.r = reach
        self.sponge = (0, 0.0) if not sponge else (int(sponge[0]), float(sponge[1]))
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.device = dev
        self.nz, self.ny, self.nx = reach.solid.shape
        self.N = reach.solid.size
        nu_lb = max(1e-6 * reach.dt / reach.dx ** 2, 2e-4)
        self.tau0, self.csmag2 = 0.5 + 3 * nu_lb, float(reach.cfg.cs) ** 2
        T = lambda a, dt: torch.from_numpy(np.ascontiguousarray(np.asarray(a).ravel()).astype(dt)).to(dev)  # noqa: E731
        self.solid = T(reach.solid, np.uint8)
        self.bedwall = T(reach.bedwall, np.uint8) if reach.bedwall is not None else None
        self.F0 = [T(a, np.float32) for a in (reach.Fx, reach.Fy, reach.Fz)]
        self.F = [torch.empty(self.N, dtype=torch.float64, device=dev) for _ in range(3)]
        cf = reach.cf if reach.cf is not None else np.zeros(reach.solid.shape, np.float32)
        self.cfw = T(np.asarray(cf, np.float32), np.float64)
        uin = (reach.uin_phys / reach.vel).astype(np.float32)
        self.uin = T(uin, np.float64)
        self.rho = torch.ones(self.N, dtype=torch.float64, device=dev)
        self.ux, self.uy, self.uz, self.uref = (torch.zeros(self.N, dtype=torch.float64, device=dev) for _ in range(4))
        # 1D-profile start (floodsim/lbm3d.py:362-364, 377-384): feq(1, (uin(y,z), 0, 0)) along x, 0 at solids
        u0 = self.uin.view(self.nz, self.ny, 1).expand(self.nz, self.ny, self.nx).reshape(-1).clone()
        u0[self.solid.bool()] = 0.0
        self.f = torch.empty(19 * self.N, dtype=torch.float64, device=dev)
        for i in range(19):
            cu = 3.0 * CX[i] * u0
            self.f[i * self.N:(i + 1) * self.N] = W64[i] * (1.0 + cu + 0.5 * cu * cu - 1.5 * u0 * u0)
        self.f2 = self.f.clone()
        self.set_force_scale(np.float32(1.0))
        self.nstep = 0
        self.t = 0.0
        self.sums, self.navg = None, 0

    def _stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def set_force_scale(self, scale):
        """Forces = float32 forces x float32 scale, in float64 (the ramp of Run3D.advance)."""
        s = self.torch.tensor(np.float32(scale), device=self.device)
        for F, F0 in zip(self.F, self.F0):
            F.copy_((F0 * s).to(self.torch.float64))

    def update_uref(self):
        if self.bedwall is None:
            return
        p = lambda a: a.data_ptr()  # noqa: E731
        nat.check(self.lib.lbm_update_uref_f64(p(self.ux), p(self.uy), p(self.solid), p(self.bedwall), p(self.uref),
                                               self.nx, self.ny, self.nz, self._stream()), "lbm_update_uref_f64")

    def step(self, n=1):
        p = lambda a: a.data_ptr()  # noqa: E731
        st = self._stream()
        for _ in range(n):
            nat.check(self.lib.lbm_step_f64(p(self.f), p(self.f2), p(self.solid), *(p(F) for F in self.F), p(self.rho),
                                            p(self.ux), p(self.uy), p(self.uz), p(self.cfw), p(self.uref),
                                            self.nx, self.ny, self.nz, self.tau0, self.csmag2, *self.sponge, st),
                      "lbm_step_f64")
            nat.check(self.lib.lbm_bc_f64(p(self.f2), p(self.solid), p(self.uin), self.nx, self.ny, self.nz, 1.0, st),
                      "lbm_bc_f64")
            self.f, self.f2 = self.f2, self.f
        self.nstep += n

    def perturb(self, rel=6e-8, seed=3):
        """Multiply the populations by 1 + rel * N(0, 1): a second float64 trajectory of the same
        case (rel = 6e-8 is half a float32 ulp), whose distance from the first is the spread the
        flow's readouts have by themselves -- the floor of any precision statement."""
        torch = self.torch
        g = torch.Generator(device=self.device).manual_seed(seed)
        self.f.mul_(1 + rel * torch.randn(self.f.shape, generator=g, device=self.device, dtype=torch.float64))
        self.f2.copy_(self.f)

    def advance(self, steps, average=False, t_avg=None):
        """`steps` steps with Run3D.advance's chunking, ramp and uref refresh; with `average`,
        the float64 sums of (rho, ux, uy, uz, |u|, ux^2) at the chunk ends with t >= t_avg
        (default: the case's own averaging start)."""
        torch, r = self.torch, self.r
        t_total = r.cfg.run_flows * r.cfg.length / max(r.V, 0.05)
        t_ramp = min(0.15 * t_total, 20.0) if r.props else 0.0
        if t_avg is None:
            t_avg = t_total * (1 - r.cfg.avg_frac)
        ramp_done = t_ramp <= 0
        if not ramp_done and self.nstep == 0:
            self.set_force_scale(np.float32(0.0))
        k = 0
        while k < steps:
            m = min(Run3D.avg_every, steps - k)
            if not ramp_done:
                f = min(self.t / t_ramp, 1.0)
                scale = np.float32(f * f * (3 - 2 * f))
                self.set_force_scale(scale)
                ramp_done = bool(scale >= 1.0)
            self.update_uref()
            self.step(m)
            k += m
            self.t += m * r.dt
            if average and self.t >= t_avg:
                sp = torch.sqrt(self.ux * self.ux + self.uy * self.uy + self.uz * self.uz)
                add = (self.rho, self.ux, self.uy, self.uz, sp, self.ux * self.ux)
                if self.sums is None:
                    self.sums = [a.clone() for a in add]
                else:
                    for s, a in zip(self.sums, add):
                        s.add_(a)
                self.navg += 1

    def fields(self, mean=False):
        """Host float64 (rho, ux, uy, uz, speed): instantaneous, or the time averages."""
        if mean:
            if not self.navg:
                raise ValueError("no averaged outputs yet")
            r, u, v, w, sp, _ = (s.cpu().numpy() / self.navg for s in self.sums)
            return r, u, v, w, sp
        r, u, v, w = (a.cpu().numpy() for a in (self.rho, self.ux, self.uy, self.uz))
        return r, u, v, w, np.sqrt(u * u + v * v + w * w)
