"""LBM3D: the reference's D3Q19 solver object (floodsim/lbm3d.py:333-418) on B200 kernels.

Same constructor, same public arrays (``f, f2, rho, ux, uy, uz, Fx, Fy, Fz, uin,
uref, cfw, solid``), same ``step(n)``, ``set_force``, ``shape3`` and
``memory_mb``, same ``TypeError`` on a force/inlet/uref array of the wrong dtype
or size.  Arrays are torch CUDA tensors.  Every step is one launch of the fused
kernel of liblbm_b200.so (``lbm_fused_step``); there is no CPU path.

Additions, all optional and off by default:

* ``uref_mode="column"`` -- the wall model's reference speed at bed/bank cells is
  the column depth-mean speed that the kernel itself refreshes at the end of
  every ``step(n)`` call (the reference's ``Run3D._update_uref``,
  floodsim/reach3d.py:412-418, fused into the sweep).  Needs ``bedwall``.
* ``force_scale`` -- scalar multiplying Fx/Fy/Fz inside the kernel (the force
  ramp of floodsim/reach3d.py:431-437 without rewriting the arrays).
* ``enable_averaging()`` / ``step(n, accumulate=True)`` -- the time-average
  sums of floodsim/reach3d.py:443-451, added by the last step of the call.
* ``storage="fp16"`` -- populations stored as 16-bit deviations from the lattice
  weights, fp16((f_i - w_i) * store_scale), collision in FP32
  (``lbm_fused_step_h``): half the population traffic of the float32 store.
  ``f``/``f2`` then hold the raw 16-bit values; ``populations()`` decodes them.
"""
from __future__ import annotations

import numpy as np

from . import _native as nat

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
OPP = np.array([0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17])
MIRZ = np.array([0, 1, 2, 3, 4, 6, 5, 7, 8, 9, 10, 13, 14, 11, 12, 17, 18, 15, 16])

AVG_FIELDS = ("ux", "uy", "uz", "rho", "sp", "uxx")
# (pipeline, cells_per_lane, warps, stages, ctas_per_sm): work lists over 128-cell row segments,
# 4 warps per CTA, as many CTAs per SM as fit
DEFAULT_TILE = (3, 4, 4, 0, 0)
# 16-bit storage: work lists over 64-cell row segments (plain segments: 8 lanes of one 16-byte
# vector of 8 cells each)
DEFAULT_TILE_FP16 = (3, 2, 4, 0, 0)
STORAGES = ("fp32", "fp16")
# |f_i - w_i| < 65504 / 2^14 ~ 4 is representable (populations of a stable lattice lie in (0, 1)),
# and every deviation above 2^-28 keeps fp16's full 11-bit significand
DEFAULT_STORE_SCALE = 2.0 ** 14


def _ptr(t):
    return ctypes_ptr(t)


def ctypes_ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


class LBM3D:
    """D3Q19 regularized-BGK + Smagorinsky solver on one CUDA device.

    solid: bool (nz, ny, nx); Fx, Fy, Fz: force per unit volume in lattice units
    (nz, ny, nx); uin: inlet velocity in lattice units (nz, ny); tau0: relaxation
    time; cs: Smagorinsky constant; cf_wall: wall friction coefficient
    tau = rho*cf*U^2 of wall-adjacent cells (nz, ny, nx), None = plain no-slip.
    ``be`` is accepted for signature compatibility (any object; a
    ``torch.device`` or an object with a ``device`` attribute picks the GPU).
    """

    engine = "cuda-b200"

    def __init__(self, be, solid, Fx, Fy, Fz, uin, tau0, cs=0.17, cf_wall=None, *, bedwall=None,
                 uref_mode="field", tile=None, device=None, storage="fp32", store_scale=DEFAULT_STORE_SCALE,
                 sponge=None):
        torch = nat.require_cuda()
        # optional outlet sponge (cols, tau_at_outlet), not in the reference: split pipeline only
        self.sponge_cols, self.sponge_tau = (0, 0.0) if not sponge else (int(sponge[0]), float(sponge[1]))
        self._torch = torch
        self.lib = nat.load()
        self.be = be
        dev = device if device is not None else getattr(be, "device", None)
        if dev is None and isinstance(be, torch.device):
            dev = be
        self.device = torch.device(dev) if dev is not None else torch.device("cuda", torch.cuda.current_device())
        shape = tuple(solid.shape)
        self.nz, self.ny, self.nx = shape
        self.N = self.nz * self.ny * self.nx
        if storage not in STORAGES:
            raise ValueError(f"storage must be one of {STORAGES}")
        self.storage = storage
        self.store_scale = float(store_scale)
        align = 8 if storage == "fp16" else 4
        self.pitch = (self.nx + align - 1) // align * align
        self.cells = self.pitch * self.ny * self.nz
        self.tau0 = float(tau0)
        self.csmag2 = float(cs * cs)
        self.rho_out = 1.0
        self.force_scale = 1.0
        self.xp = torch
        self.nstep = 0
        self.navg = 0
        self.overlap = False
        self.tile = self._tile_of(tile or (DEFAULT_TILE_FP16 if storage == "fp16" else DEFAULT_TILE))
        self._wl = None
        if uref_mode not in ("field", "column"):
            raise ValueError("uref_mode must be 'field' or 'column'")
        if uref_mode == "column" and bedwall is None:
            raise ValueError("uref_mode='column' needs the bedwall mask")
        self.uref_mode = uref_mode

        d, f32 = self.device, torch.float32
        self._solid_np = None if isinstance(solid, torch.Tensor) else np.asarray(solid, bool)
        self._solid = self._pitched(solid, torch.uint8, pad=1)
        self._bedwall = None if bedwall is None else self._pitched(bedwall, torch.uint8)
        self._F = [self._pitched(a, f32) for a in (Fx, Fy, Fz)]
        self._cfw = (torch.zeros(self.cells, dtype=f32, device=d) if cf_wall is None else self._pitched(cf_wall, f32))
        self._uref = torch.zeros(self.cells, dtype=f32, device=d)
        if isinstance(uin, torch.Tensor):
            self._uin = uin.to(d, f32, non_blocking=True).reshape(-1).contiguous()
        else:
            self._uin = torch.as_tensor(np.ascontiguousarray(np.asarray(uin, np.float32)).ravel(), device=d)
        self._rho = torch.ones(self.cells, dtype=f32, device=d)
        self._ux = torch.zeros(self.cells, dtype=f32, device=d)
        self._uy = torch.zeros(self.cells, dtype=f32, device=d)
        self._uz = torch.zeros(self.cells, dtype=f32, device=d)
        self._colU = torch.zeros(self.ny * self.pitch, dtype=f32, device=d)
        self._flags = torch.zeros(self.cells, dtype=torch.int32, device=d)
        self._status = torch.zeros(4, dtype=torch.int32, device=d)
        self._avg = None
        self._body_scratch = None
        self._bad = {}
        pop_dtype = torch.float16 if storage == "fp16" else f32
        self.f = torch.empty(19 * self.cells, dtype=pop_dtype, device=d)
        self.f2 = torch.empty(19 * self.cells, dtype=pop_dtype, device=d)
        self._flag_versions = None
        self._build_flags()
        if storage == "fp16":
            nat.check(self.lib.lbm_init_equilibrium_h(self._lattice_ref(), ctypes_ptr(self.f), self.store_scale,
                                                      self._stream()), "lbm_init_equilibrium_h")
        else:
            nat.check(self.lib.lbm_init_equilibrium(self._lattice_ref(), ctypes_ptr(self.f), self._stream()),
                      "lbm_init_equilibrium")
        self.f2.copy_(self.f)

    # ------------------------------------------------------------------ layout helpers
    def _pitched(self, a, dtype, pad=0):
        """(nz,ny,nx) array (NumPy, or a torch tensor on the host -- pinned for an asynchronous
        copy -- or on the device) -> flat device tensor with x pitch `self.pitch` (padding = pad)."""
        torch = self._torch
        if isinstance(a, torch.Tensor):
            if a.numel() != self.N:
                raise TypeError(f"LBM3D: array of size {a.numel()} does not match the lattice ({self.N} cells)")
            t = a.to(self.device, non_blocking=True).reshape(self.nz, self.ny, self.nx).to(dtype)
            if self.pitch != self.nx:
                b = torch.full((self.nz, self.ny, self.pitch), pad, dtype=dtype, device=self.device)
                b[..., :self.nx] = t
                t = b
            return t.reshape(-1).contiguous()
        a = np.asarray(a)
        if a.dtype == bool:
            a = a.astype(np.uint8)
        if a.size != self.N:
            raise TypeError(f"LBM3D: array of size {a.size} does not match the lattice ({self.N} cells)")
        a = a.reshape(self.nz, self.ny, self.nx)
        if self.pitch != self.nx:
            b = np.full((self.nz, self.ny, self.pitch), pad, dtype=a.dtype)
            b[..., :self.nx] = a
            a = b
        return torch.as_tensor(np.ascontiguousarray(a).ravel(), dtype=dtype, device=self.device)

    def _view(self, t):
        """Flat (N,) reference-layout view of a pitched per-cell tensor (a copy when pitch != nx)."""
        if self.pitch == self.nx:
            return t
        return t.view(self.nz, self.ny, self.pitch)[..., :self.nx].reshape(-1)

    def _stream(self):
        return self._torch.cuda.current_stream(self.device).cuda_stream

    def _lattice(self) -> nat.Lattice:
        L = nat.Lattice()
        L.nx, L.ny, L.nz, L.pitch, L.cells = self.nx, self.ny, self.nz, self.pitch, self.cells
        L.tau0, L.csmag2, L.rho_out, L.force_scale = self.tau0, self.csmag2, self.rho_out, self.force_scale
        L.flags = ctypes_ptr(self._flags)
        L.Fx, L.Fy, L.Fz = (ctypes_ptr(a) for a in self._F)
        L.cfw, L.uref, L.uin = ctypes_ptr(self._cfw), ctypes_ptr(self._uref), ctypes_ptr(self._uin)
        L.rho, L.ux, L.uy, L.uz = (ctypes_ptr(a) for a in (self._rho, self._ux, self._uy, self._uz))
        L.colU, L.avg, L.status = ctypes_ptr(self._colU), ctypes_ptr(self._avg), ctypes_ptr(self._status)
        if self._wl is not None:
            lists, counts, v = self._wl
            L.rows_plain, L.rows_solid, L.rows_special, L.rows_edge = (ctypes_ptr(a) for a in lists)
            L.n_plain, L.n_solid, L.n_special, L.n_edge = counts
            L.list_cells_per_lane = v
        L.sponge_cols, L.sponge_tau = self.sponge_cols, self.sponge_tau
        return L

    def _lattice_ref(self):
        import ctypes
        self._lat_keep = self._lattice()
        return ctypes.byref(self._lat_keep)

    def _versions(self):
        return tuple(t._version for t in (*self._F, self._cfw))

    def _build_flags(self):
        nat.check(self.lib.lbm_build_flags(self._lattice_ref(), ctypes_ptr(self._solid), ctypes_ptr(self._bedwall),
                                           ctypes_ptr(self._flags), self._stream()), "lbm_build_flags")
        self._flag_versions = self._versions()
        self._wl = None
        if self.tile.pipeline == nat.PIPE_SPLIT:
            self._build_worklists()

    def _build_worklists(self):
        """Plain / solid / special / edge row-segment lists of the split pipeline (from the flags)."""
        torch = self._torch
        v = self.tile.cells_per_lane
        seg = 32 * v
        n = (self.pitch + seg - 1) // seg * self.ny * self.nz
        scratch = torch.empty(n, dtype=torch.uint8, device=self.device)
        lists = [torch.empty(n, dtype=torch.int32, device=self.device) for _ in range(4)]
        counts = torch.zeros(4, dtype=torch.int32, device=self.device)
        self._wl = None
        nat.check(self.lib.lbm_build_worklists(self._lattice_ref(), v, ctypes_ptr(scratch), *(ctypes_ptr(a) for a in lists),
                                               ctypes_ptr(counts), self._stream()), "lbm_build_worklists")
        c = tuple(int(x) for x in counts.cpu())
        self._wl = ([a[:max(k, 1)].clone() for a, k in zip(lists, c)], c, v)

    def _tile_of(self, tile):
        """nat.Tile of a 5-tuple (pipeline, cells_per_lane, warps, stages, ctas_per_sm), or of a 6-tuple
        whose last entry sets `overlap` (LBM_STEP_OVERLAP: the edge and special kernels of the split
        pipeline run on a side stream beside the plain kernel, ctas_per_sm bounding the plain kernel)."""
        tile = tuple(tile)
        self.overlap = len(tile) == 6 and bool(tile[5])
        return nat.Tile(*tile[:5])

    def tile_key(self):
        """The launch shape as autotune candidates spell it: 5 entries, or 6 with overlap on."""
        return self.tile.key() + ((1,) if self.overlap else ())

    def set_tile(self, tile):
        """Change the launch shape (pipeline, cells_per_lane, warps, stages, ctas_per_sm[, overlap])."""
        self.tile = self._tile_of(tile)
        self._build_flags()

    def worklist_counts(self):
        """(plain, solid, special, edge) row-segment counts of the split pipeline, or None."""
        return None if self._wl is None else self._wl[1]

    # ------------------------------------------------------------------ public arrays
    @property
    def solid(self):
        return self._view(self._solid)

    def layer(self, name, z=-1):
        """One z layer of a field ("rho", "ux", "uy" or "uz") as a (ny, nx) view of the device
        field, without the copy of the whole field that the flat reference-layout attributes
        make when the x pitch exceeds nx (the lid level, for instance, needs the top layer only)."""
        if name not in ("rho", "ux", "uy", "uz"):
            raise ValueError(f"layer: unknown field {name!r}")
        return getattr(self, "_" + name).view(self.nz, self.ny, self.pitch)[z, :, :self.nx]

    @property
    def rho(self):
        return self._view(self._rho)

    @property
    def ux(self):
        return self._view(self._ux)

    @property
    def uy(self):
        return self._view(self._uy)

    @property
    def uz(self):
        return self._view(self._uz)

    @property
    def uin(self):
        return self._uin

    @property
    def cfw(self):
        return self._view(self._cfw)

    @property
    def flags(self):
        return self._view(self._flags)

    def _set_cell_array(self, name, buf, a):
        """Copy a caller-assigned per-cell array into `buf`; a wrong dtype or size is
        remembered and reported by the next step(), as the reference does."""
        torch = self._torch
        size = a.numel() if isinstance(a, torch.Tensor) else np.asarray(a).size
        dtype_ok = (a.dtype == torch.float32) if isinstance(a, torch.Tensor) else (np.asarray(a).dtype == np.float32)
        if not dtype_ok or size != self.N:
            self._bad[name] = (a.dtype, size)
            return
        self._bad.pop(name, None)
        if isinstance(a, torch.Tensor):
            src = a.reshape(self.nz, self.ny, self.nx).to(self.device)
        else:
            src = torch.as_tensor(np.ascontiguousarray(np.asarray(a)).reshape(self.nz, self.ny, self.nx),
                                  device=self.device)
        buf.view(self.nz, self.ny, self.pitch)[..., :self.nx].copy_(src)

    Fx = property(lambda self: self._view(self._F[0]),
                  lambda self, a: self._set_cell_array("Fx", self._F[0], a))
    Fy = property(lambda self: self._view(self._F[1]),
                  lambda self, a: self._set_cell_array("Fy", self._F[1], a))
    Fz = property(lambda self: self._view(self._F[2]),
                  lambda self, a: self._set_cell_array("Fz", self._F[2], a))

    @property
    def uref(self):
        if self.uref_mode == "column":
            torch = self._torch
            col = self._colU.view(1, self.ny, self.pitch).expand(self.nz, self.ny, self.pitch)
            bw = self._bedwall.view(self.nz, self.ny, self.pitch).bool()
            full = torch.where(bw, col, torch.zeros((), device=self.device))
            return full[..., :self.nx].reshape(-1)
        return self._view(self._uref)

    @uref.setter
    def uref(self, a):
        self.uref_mode = "field"
        self._set_cell_array("uref", self._uref, a)

    def set_force(self, Fx, Fy, Fz):
        """floodsim/lbm3d.py:386-388: any dtype, converted to float32."""
        torch = self._torch
        for k, a in enumerate((Fx, Fy, Fz)):
            t = a.to(self.device, torch.float32) if isinstance(a, torch.Tensor) else \
                torch.as_tensor(np.asarray(a, np.float32), device=self.device)
            self._set_cell_array("F" + "xyz"[k], self._F[k], t)

    def enable_averaging(self):
        """Allocate the six time-average sums (ux, uy, uz, rho, |u|, ux^2), zeroed."""
        if self._avg is None:
            self._avg = self._torch.zeros(6 * self.cells, dtype=self._torch.float32, device=self.device)
        else:
            self._avg.zero_()
        self.navg = 0

    def profile_sums(self, mean=True):
        """Float64 cross-section sums per x station (lbm_profiles), in lattice units, as host
        arrays: q, uxx, drho, mass, n_fluid, top_n, top_drho, top_ux, umax (each (nx,)) and
        bed_speed2 ((ny, nx)).  mean=True reduces the time averages (needs averaging enabled
        and at least one accumulated output), else the current fields."""
        torch = self._torch
        use_avg = mean and self._avg is not None and self.navg > 0
        if mean and not use_avg:
            raise ValueError("profile_sums(mean=True) needs accumulated time averages")
        L = self._lattice()
        if not use_avg:
            L.avg = None
        import ctypes
        ref = ctypes.byref(L)
        n_scr = int(self.lib.lbm_profiles_scratch_doubles(ref))
        if n_scr < 0:
            nat.check(n_scr, "lbm_profiles_scratch_doubles")
        f64 = torch.float64
        prof = torch.empty(len(nat.PROFILE_FIELDS) * self.nx, dtype=f64, device=self.device)
        sp2 = torch.empty(self.ny * self.nx, dtype=f64, device=self.device)
        scratch = torch.empty(max(n_scr, 1), dtype=f64, device=self.device)
        inv = 1.0 / self.navg if use_avg else 1.0
        nat.check(self.lib.lbm_profiles(ref, inv, ctypes_ptr(prof), ctypes_ptr(sp2), ctypes_ptr(scratch),
                                        self._stream()), "lbm_profiles")
        p = prof.view(len(nat.PROFILE_FIELDS), self.nx).cpu().numpy()
        out = {k: p[i] for i, k in enumerate(nat.PROFILE_FIELDS)}
        out["bed_speed2"] = sp2.view(self.ny, self.nx).cpu().numpy()
        return out

    def body_forces(self, body, nbody):
        """Float64 force sums from the current state (lbm_body_forces): the momentum-exchange force
        on each body of `body` (uint8 (nz, ny, nx) or a pitched device tensor; body k's cells hold
        k, 1..nbody) for the next step's bounce-back, and the body force the step applies.
        Returns (forces (nbody, 3), applied (3,)) as float64 host arrays in lattice units."""
        torch = self._torch
        import ctypes
        if nbody == 0:
            body = None
        elif not isinstance(body, torch.Tensor) or body.numel() != self.cells:
            body = self._pitched(body, torch.uint8)
        if self._body_scratch is None or self._body_scratch[0] != nbody:
            n = int(self.lib.lbm_body_forces_scratch_doubles(int(nbody)))
            if n < 0:
                nat.check(n, "lbm_body_forces_scratch_doubles")
            self._body_scratch = (nbody, torch.empty(n, dtype=torch.float64, device=self.device))
        out = torch.empty(3 * nbody + 3, dtype=torch.float64, device=self.device)
        L = self._lattice()
        mode = nat.STEP_UREF_COLUMN if self.uref_mode == "column" else 0
        scr = ctypes_ptr(self._body_scratch[1])
        if self.storage == "fp16":
            rc = self.lib.lbm_body_forces_h(ctypes.byref(L), ctypes_ptr(self.f), self.store_scale, ctypes_ptr(body),
                                            int(nbody), mode, ctypes_ptr(out), scr, self._stream())
        else:
            rc = self.lib.lbm_body_forces(ctypes.byref(L), ctypes_ptr(self.f), ctypes_ptr(body), int(nbody), mode,
                                          ctypes_ptr(out), scr, self._stream())
        nat.check(rc, "lbm_body_forces")
        o = out.cpu().numpy()
        return o[:3 * nbody].reshape(nbody, 3), o[3 * nbody:]

    def avg_sum(self, name):
        """Flat (N,) view of one time-average sum (divide by navg for the mean)."""
        k = AVG_FIELDS.index(name)
        return self._view(self._avg[k * self.cells:(k + 1) * self.cells])

    # ------------------------------------------------------------------ stepping
    def step(self, n=1, accumulate=False):
        """Advance n time steps (floodsim/lbm3d.py:390-412): one fused launch each."""
        if self._bad:
            name, (dt, size) = next(iter(self._bad.items()))
            raise TypeError(f"LBM3D: force/inlet arrays must be float32 of the correct size (got {dt}, {size})")
        if self._uin.dtype != self._torch.float32 or self._uin.numel() != self.ny * self.nz:
            raise TypeError(f"LBM3D: force/inlet arrays must be float32 of the correct size "
                            f"(got {self._uin.dtype}, {self._uin.numel()})")
        if accumulate and self._avg is None:
            self.enable_averaging()
        if self._versions() != self._flag_versions:
            self._build_flags()
        lat = self._lattice_ref()
        st = self._stream()
        col = nat.STEP_UREF_COLUMN if self.uref_mode == "column" else 0
        if self.overlap and self.tile.pipeline == nat.PIPE_SPLIT:
            col |= nat.STEP_OVERLAP
        tile = self.tile
        half = self.storage == "fp16"
        for k in range(n):
            mode = col
            if k == n - 1:
                mode |= nat.STEP_OUTPUT | (nat.STEP_ACCUMULATE if accumulate else 0)
            if half:
                nat.check(self.lib.lbm_fused_step_h(lat, ctypes_ptr(self.f), ctypes_ptr(self.f2), self.store_scale,
                                                    mode, tile, st), "lbm_fused_step_h")
            else:
                nat.check(self.lib.lbm_fused_step(lat, ctypes_ptr(self.f), ctypes_ptr(self.f2), mode, tile, st),
                          "lbm_fused_step")
            self.f, self.f2 = self.f2, self.f
        if n > 0 and accumulate:
            self.navg += 1
        self.nstep += n

    def status(self) -> int:
        """Device status word (bit 0: a non-finite or non-positive density was written). Synchronizes."""
        return int(self._status[0].item())

    # ------------------------------------------------------------------ reference helpers
    def shape3(self, a):
        return a.reshape(self.nz, self.ny, self.nx)

    def memory_mb(self):
        pop = 2 if self.storage == "fp16" else 4
        return self.N * (19 * 2 * pop + 4 * 10 + 1) / 1e6

    def populations_device(self):
        """Current populations as a float32 device tensor in the pitched layout f[i*cells + c]."""
        if self.storage != "fp16":
            return self.f
        out = self._torch.empty(19 * self.cells, dtype=self._torch.float32, device=self.device)
        nat.check(self.lib.lbm_unpack_populations(self._lattice_ref(), ctypes_ptr(self.f), ctypes_ptr(out),
                                                  self.store_scale, self._stream()), "lbm_unpack_populations")
        return out

    def load_populations(self, f):
        """Replace the state by float32 populations (device tensor, pitched layout, 19*cells)."""
        torch = self._torch
        if f.dtype != torch.float32 or f.numel() != 19 * self.cells:
            raise TypeError("load_populations: float32 tensor of 19*cells elements expected")
        f = f.to(self.device).contiguous()
        if self.storage == "fp16":
            nat.check(self.lib.lbm_pack_populations(self._lattice_ref(), ctypes_ptr(f), ctypes_ptr(self.f),
                                                    self.store_scale, self._stream()), "lbm_pack_populations")
        else:
            self.f.copy_(f)
        self.f2.copy_(self.f)

    def populations(self):
        """Current populations as a host float32 array in the reference layout f[i*N + c]."""
        f = self.populations_device().view(19, self.nz, self.ny, self.pitch)[..., :self.nx]
        return f.reshape(-1).cpu().numpy()
