"""3D reach set-up, time loop and readouts around the B200 solver.

Host-side counterpart of the reference's floodsim/reach3d.py, with the same public
names, arguments and results:

* ``BoatType``, ``BOAT_TYPES``, ``boat_type``, ``Fleet``, ``ReachConfig``, ``Reach``
  (reach3d.py:24-190) -- boat physics and case description;
* ``bed_level``, ``auto_dx``, ``build_reach`` (reach3d.py:142-297) -- lattice, solid
  mask, 1/7-power inlet profile, hulls, actuator disks and jets, time step, lattice
  forces; ``wall_cf``, ``log_cf``, ``manning_ks`` (reach3d.py:305-343) -- Manning
  bed/bank and log-law hull friction; the arrays are bit-identical to the
  reference's (tests/test_reach_builder.py);
* ``Run3D`` (reach3d.py:378-497) -- the time loop on ``LBM3D``: 20-step chunks,
  smoothstep force ramp, column-mean wall-model speed and time averages, here all
  done inside the fused kernel (a scalar force scale, the kernel's column-mean
  refresh and its accumulation epilogue) instead of by separate array passes;
* ``profiles``, ``compare`` (reach3d.py:545-618) -- water level, discharge, bed
  shear, momentum flux and the boat-versus-base comparison.

The numeric expressions of the builder are written so that NumPy performs the same
operations in the same dtypes as the reference (float32 arrays times Python floats
stay float32, for instance): that is what makes the arrays identical.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field, replace

import numpy as np
from scipy.ndimage import binary_dilation, distance_transform_edt

from .geometry import Section
from .lbm3d import LBM3D

G = 9.81
RHO = 1000.0
N_SLOSH = 10          # pressure-wave round trips the averaging window must hold
F_LB_MAX = 1.5e-3     # largest lattice body force per cell before dt is reduced


# ------------------------------------------------------------------------------ boats
@dataclass
class BoatType:
    key: str
    name: str
    hull_L: float          # hull length (m)
    hull_B: float          # hull beam (m)
    draft: float           # draft (m)
    n_props: int           # propellers (or nozzles) per boat
    prop_D: float          # propeller diameter (m)
    prop_depth: float      # depth of the propeller centre below the surface (m)
    tilt_deg: float        # downward shaft tilt (deg, 0 = horizontal)
    prop_x: float          # propeller position behind the stern (m; negative = under the hull)
    prop_spacing: float    # transverse spacing of the propellers (m)
    power_kW: float        # shaft power per propeller (kW)
    merit: float = 0.6     # figure of merit
    thrust_N: float = 0.0  # prescribed thrust (0 = from the power)
    note: str = ""
    jet_bar: float = 0.0   # nozzle pressure (bar); 0 = propeller
    spread_deg: float = 0.0  # jets split into yaws -spread, 0, +spread

    @property
    def is_jet(self) -> bool:
        return self.jet_bar > 0

    def thrust(self) -> float:
        """Thrust per propeller or nozzle (N): actuator disk T = (2 rho A (eta P)^2)^(1/3),
        or for a jet, with eta P = m v^2 / 2 and T = m v, T = 2 eta P / v."""
        if self.thrust_N > 0:
            return self.thrust_N
        if self.is_jet:
            return 2 * self.merit * self.power_kW * 1000 / self.jet_speed()
        disk = math.pi * self.prop_D ** 2 / 4
        return (2 * RHO * disk * (self.merit * self.power_kW * 1000) ** 2) ** (1 / 3)

    def jet_speed(self) -> float:
        """Outflow speed (m/s): nozzle sqrt(2 dp / rho); propeller ~ 2 sqrt(T / (2 rho A))."""
        if self.is_jet:
            return math.sqrt(2 * self.jet_bar * 1e5 / RHO)
        disk = max(math.pi * self.prop_D ** 2 / 4, 1e-6)
        return 2 * math.sqrt(self.thrust() / (2 * RHO * disk))

    def outlet_D(self) -> float:
        """Propeller diameter, or the nozzle diameter that carries the thrust (T = rho A v^2)."""
        if self.is_jet:
            v = self.jet_speed()
            return math.sqrt(4 * self.thrust() / (math.pi * RHO * v * v))
        return self.prop_D


# The reference's boat catalogue (floodsim/reach3d.py:75-93): same keys and parameters.
BOAT_TYPES = [
    BoatType("longtail", "long-tail boat", 9.0, 1.6, 0.35, 1, 0.30, 0.35, 12, 2.5, 0, 75),
    BoatType("outboard", "outboard boat", 7.0, 2.4, 0.5, 1, 0.36, 0.6, 0, 0.3, 0, 110),
    BoatType("tug", "tug / push boat", 16.0, 5.0, 1.8, 2, 1.2, 1.6, 0, -1.0, 2.4, 300),
    BoatType("pontoon", "float-mounted pusher", 6.0, 4.0, 0.5, 1, 1.6, 1.3, 0, 0.5, 0, 30),
    BoatType("jet_hp", "high-pressure jets (100 bar)", 6.0, 4.0, 0.5, 4, 0.0, 1.2, 0, 0.3, 0.8, 25,
             merit=0.7, jet_bar=100),
    BoatType("jet_mp", "medium-pressure jets (10 bar)", 6.0, 4.0, 0.5, 4, 0.0, 1.2, 0, 0.3, 0.8, 25,
             merit=0.7, jet_bar=10),
    BoatType("curtain", "low-speed water curtain", 6.0, 6.0, 0.5, 4, 0.0, 1.3, 0, 0.3, 1.4, 25,
             merit=0.7, jet_bar=0.045),
    BoatType("custom", "custom", 10.0, 3.0, 0.8, 1, 0.8, 1.0, 0, 0.5, 0, 100),
]


def boat_type(key: str) -> BoatType:
    for b in BOAT_TYPES:
        if b.key == key:
            return replace(b)
    raise KeyError(key)


@dataclass
class Fleet:
    boat: BoatType
    rows: int = 1             # rows along the stream
    per_row: int = 3          # boats abreast in a row
    row_spacing: float = 30.0
    x_first: float = 40.0     # bow of the first row, from the inlet (m)
    enabled: bool = True

    @property
    def n_boats(self):
        return self.rows * self.per_row if self.enabled else 0

    def total_thrust(self):
        return self.n_boats * self.boat.n_props * self.boat.thrust()

    def total_power(self):
        return self.n_boats * self.boat.n_props * self.boat.power_kW

    def label(self):
        if not self.enabled or self.n_boats == 0:
            return "no boats"
        return f"{self.boat.name} {self.rows}x{self.per_row}"


@dataclass
class ReachConfig:
    length: float = 150.0      # reach length (m)
    dx: float = 0.0            # cell size (m), 0 = from max_cells
    max_cells: int = 2_000_000
    fp_max: float = 40.0       # floodplain width kept in the domain per side (m)
    u_lb: float = 0.14         # largest lattice velocity (Mach control)
    cs: float = 0.17           # Smagorinsky constant
    run_flows: float = 1.0     # simulated time = run_flows * length / mean speed
    avg_frac: float = 0.4      # trailing fraction of the run that is time-averaged
    spacing_km: float = 1.0    # spacing of boat groups along the river (discharge estimate)
    tau_crit: float = 2.0      # critical bed shear stress (N/m^2)
    wall_model: bool = True    # Manning bed/bank + log-law hull friction; False = plain no-slip
    hull_ks: float = 0.002     # hull roughness (m)


# ------------------------------------------------------------------------------ geometry
def bed_level(yy, sec: Section):
    """Bed elevation across the section at lateral positions yy (m from the centre line)."""
    a = np.abs(yy)
    half_b, half_top = sec.B / 2, sec.Tb / 2
    if sec.z > 0:
        bank = np.minimum((a - half_b) / sec.z, sec.Hb)
    else:
        bank = np.where(a > half_b, sec.Hb, 0.0)
    return np.where(a <= half_b, 0.0, np.where(a <= half_top, bank, sec.Hb))


@dataclass
class Reach:
    sec: Section
    cfg: ReachConfig
    fleet: Fleet
    h: float
    Q: float
    S: float
    dx: float
    dt: float
    nx: int
    ny: int
    nz: int
    y: np.ndarray
    zc: np.ndarray
    solid: np.ndarray
    uin_phys: np.ndarray
    Fx: np.ndarray
    Fy: np.ndarray
    Fz: np.ndarray
    cf: np.ndarray = None          # wall friction coefficient of wall-adjacent fluid cells
    bedwall: np.ndarray = None     # bed/bank wall cells (reference speed = column mean)
    hulls: list = field(default_factory=list)   # (x0, x1, y0, y1, z0, z1)
    props: list = field(default_factory=list)   # dict(x, y, z, D, Deff, tilt, yaw, T, Vjet, cells)
    notes: list = field(default_factory=list)
    W: float = 0.0
    A: float = 0.0
    V: float = 0.0
    body: np.ndarray = None        # uint8 (nz, ny, nx): hull k's solid cells hold k + 1 (0 elsewhere)

    @property
    def vel(self):
        """Lattice velocity -> m/s."""
        return self.dx / self.dt

    @property
    def x(self):
        return (np.arange(self.nx) + 0.5) * self.dx

    @property
    def cells(self):
        return self.nx * self.ny * self.nz

    def eta_from_rho(self, rho):
        """Rigid-lid pressure -> equivalent water level (m)."""
        return (rho - 1.0) / 3.0 * self.vel ** 2 / G


def auto_dx(L, Wd, h, cfg: ReachConfig):
    budget = (L * Wd * h / cfg.max_cells) ** (1 / 3)
    return float(min(max(budget, h / 40), max(h / 8, budget)))


def _inlet_profile(fluid2, dx, wall_model):
    """1/7-power profile from the distance to bed and banks, the lid mirrored (no wall),
    column means rescaled to h_col^(2/3) under the wall model (reach3d.py:218-229)."""
    mirrored = np.concatenate([fluid2, fluid2[::-1]], axis=0)
    dist = distance_transform_edt(mirrored)[: fluid2.shape[0]] * dx
    prof = np.where(fluid2, np.maximum(dist, 0.5 * dx) ** (1 / 7), 0.0)
    if wall_model:
        ncol = fluid2.sum(0)
        cmean = np.where(ncol > 0, prof.sum(0) / np.maximum(ncol, 1), 1.0)
        prof = prof / cmean[None, :] * (np.maximum(ncol, 1) * dx) ** (2 / 3)
        prof = np.where(fluid2, prof, 0.0)
    return prof


def _carve_hull(solid, Xc, y, zc, x0, x1, yb, hull_L, hull_B, z_keel):
    """Box hull with a bow tapering to 35 % of the beam over the first quarter (reach3d.py:246-257)."""
    in_x = (Xc >= x0) & (Xc <= x1)
    taper = np.clip((Xc[in_x] - x0) / (0.25 * hull_L), 0.35, 1.0)
    below = zc >= z_keel
    for jx, fr in zip(np.flatnonzero(in_x), taper):
        across = np.abs(y - yb) <= hull_B / 2 * fr
        solid[np.ix_(below, across, [jx])] = True


def _add_prop(Fx, Fy, Fz, solid, Xc, y, zc, dx, xp, yp, zp, D, tilt, T, yaw=0.0):
    """Spread thrust T uniformly over a disk of cells (at least 3 cells across, same total
    thrust); tilt = downward angle, yaw = horizontal deflection towards +y (reach3d.py:346-374)."""
    Deff = max(D, 3 * dx)
    t, w = math.radians(tilt), math.radians(yaw)
    ax, ay, az = math.cos(t) * math.cos(w), math.cos(t) * math.sin(w), -math.sin(t)
    reach_r = Deff / 2 + 2 * dx
    ix = np.flatnonzero(np.abs(Xc - xp) <= reach_r)
    iy = np.flatnonzero(np.abs(y - yp) <= reach_r)
    iz = np.flatnonzero(np.abs(zc - zp) <= reach_r)
    X, Yy, Z = np.meshgrid(Xc[ix] - xp, y[iy] - yp, zc[iz] - zp, indexing="ij")
    axial = X * ax + Yy * ay + Z * az
    rx, ry, rz = X - axial * ax, Yy - axial * ay, Z - axial * az
    radial = np.sqrt(rx * rx + ry * ry + rz * rz)
    disk = (np.abs(axial) <= dx * 0.75) & (radial <= Deff / 2)
    disk &= ~solid[np.ix_(iz, iy, ix)].transpose(2, 1, 0)
    ncell = int(disk.sum())
    if ncell == 0:
        return dict(x=xp, y=yp, z=zp, D=D, Deff=Deff, tilt=tilt, yaw=yaw, T=0.0, Vjet=0.0, cells=0)
    per_cell = T / (ncell * dx ** 3)                     # N/m^3
    load = np.zeros(disk.shape, np.float32)
    load[disk] = per_cell
    load = load.transpose(2, 1, 0)                       # (z, y, x)
    box = np.ix_(iz, iy, ix)
    Fx[box] += load * ax
    Fy[box] += load * ay
    Fz[box] += load * az
    area = math.pi * Deff ** 2 / 4
    return dict(x=xp, y=yp, z=zp, D=D, Deff=Deff, tilt=tilt, yaw=yaw, T=T, cells=ncell,
                Vjet=2 * math.sqrt(T / (2 * RHO * area)))


def _place_fleet(fleet, sec, h, cfg, solid, Fx, Fy, Fz, Xc, y, zc, dx, notes):
    """Hulls and propellers/jets of every boat (reach3d.py:238-276)."""
    hulls, props = [], []
    b = fleet.boat
    usable = (sec.B + 2 * sec.z * min(h, sec.Hb)) * 0.9
    if b.draft >= h * 0.9:
        notes.append(f"draft {b.draft:g} m is close to the depth {h:g} m: reduced to {0.6 * h:.2f} m")
    draft = min(b.draft, 0.6 * h)
    D = b.outlet_D()
    yaws = (-b.spread_deg, 0.0, b.spread_deg) if b.spread_deg > 0 else (0.0,)
    for r in range(fleet.rows):
        xb = fleet.x_first + r * fleet.row_spacing
        for k in range(fleet.per_row):
            yb = -usable / 2 + (k + 0.5) * usable / fleet.per_row
            x0, x1 = xb, xb + b.hull_L
            hulls.append((x0, x1, yb - b.hull_B / 2, yb + b.hull_B / 2, h - draft, h))
            _carve_hull(solid, Xc, y, zc, x0, x1, yb, b.hull_L, b.hull_B, h - draft)
            for p in range(b.n_props):
                yp = yb + (p - (b.n_props - 1) / 2) * b.prop_spacing
                depth = b.prop_depth
                if depth > h - 0.6 * D:
                    depth = max(h - 0.6 * D, 0.5 * D)
                    notes.append(f"propeller/nozzle below the bed: raised to {depth:.2f} m")
                if b.prop_x < 0 and depth < draft + 0.5 * D:
                    depth = min(draft + 0.5 * D, h - 0.5 * D)
                xp = x1 + b.prop_x
                T = b.thrust()
                for yaw in yaws:
                    pr = _add_prop(Fx, Fy, Fz, solid, Xc, y, zc, dx, xp, yp, h - depth, D,
                                   b.tilt_deg, T / len(yaws), yaw)
                    if b.is_jet:       # the jet leaves at its pressure speed (sets dt via Mach)
                        pr["Vjet"] = min(b.jet_speed(), pr["Vjet"] * 4)
                    props.append(pr)
    return hulls, props


def _time_step(cfg, dx, nx, V, uin, props, Fx, Fy, Fz, fmax=None):
    """dt from Mach (u_lb), the slosh period of the averaging window and the lattice force
    limit (reach3d.py:278-293); `fmax` (the largest |F|, float32) when the forces are not
    dense arrays."""
    Vmax_in = float(uin.max())
    Ujet = 0.8 * max([p["Vjet"] for p in props], default=0.0) + V
    Umax = max(1.6 * Vmax_in, Ujet, 0.2)
    dt = cfg.u_lb * dx / Umax
    t_win = cfg.run_flows * cfg.length / max(V, 0.05) * cfg.avg_frac
    dt = float(min(dt, t_win * dx / (N_SLOSH * 2 * math.sqrt(3) * nx * dx)))
    if fmax is None:
        fmax = float(np.sqrt(Fx ** 2 + Fy ** 2 + Fz ** 2).max()) if props else 0.0
    elif not props:
        fmax = 0.0
    if fmax > 0 and fmax * dt * dt / (RHO * dx) > F_LB_MAX:
        dt = math.sqrt(F_LB_MAX * RHO * dx / fmax)
    return dt


def lattice_grid(sec: Section, h: float, cfg: ReachConfig):
    """The reference's grid rule (floodsim/reach3d.py:204-209), allocating nothing: floodplain
    width fp, top width Wtop, the cell size dx adjusted so the surface falls on a cell face,
    and the lattice (nx, ny, nz) = (round(L/dx), ceil(Wtop/dx) + 2, round(h/dx))."""
    fp = min(sec.Bf, cfg.fp_max) if h > sec.Hb else 0.0
    Wtop = (sec.B + 2 * sec.z * min(h, sec.Hb)) + 2 * fp
    dx = cfg.dx if cfg.dx > 0 else auto_dx(cfg.length, Wtop, h, cfg)
    nz = max(int(round(h / dx)), 4)
    dx = h / nz
    ny = int(math.ceil(Wtop / dx)) + 2
    nx = max(int(round(cfg.length / dx)), 16)
    return fp, Wtop, dx, nx, ny, nz


def build_reach(sec: Section, h: float, Q: float, S: float, fleet: Fleet, cfg: ReachConfig,
                bed_bumps=None) -> Reach:
    """Lattice and inputs of one case (floodsim/reach3d.py:201-297).

    bed_bumps: optional callable (x centres, y centres) -> (ny, nx) bed elevation added to
    the section's bed (m); the bed is then three-dimensional and the inlet profile is taken
    on the x = 0 cross-section.  Without it the reach is the reference's extruded section.
    """
    notes = []
    fp, Wtop, dx, nx, ny, nz = lattice_grid(sec, h, cfg)
    y = (np.arange(ny) - ny / 2 + 0.5) * dx
    zc = (np.arange(nz) + 0.5) * dx
    zb = bed_level(y, sec)
    outside = np.abs(y) > Wtop / 2
    if bed_bumps is None:
        sol2 = (zc[:, None] < zb[None, :]) | outside[None, :]
        bed = sol2
        solid = np.broadcast_to(sol2[:, :, None], (nz, ny, nx)).copy()
    else:
        zb3 = zb[:, None] + bed_bumps((np.arange(nx) + 0.5) * dx, y)
        bed = (zc[:, None, None] < zb3[None, :, :]) | outside[None, :, None]
        sol2 = bed[:, :, 0]
        solid = bed.copy()
    if fp > 0 and sec.Bf > fp:
        notes.append(f"floodplain modelled to {fp:g} m per side (the domain edge is a wall)")

    fluid2 = ~sol2
    prof = _inlet_profile(fluid2, dx, cfg.wall_model)
    A = fluid2.sum() * dx * dx
    V = Q / A
    uin = prof * (V * fluid2.sum() / prof.sum())

    Fx = np.zeros(solid.shape, np.float32)
    Fy = np.zeros(solid.shape, np.float32)
    Fz = np.zeros(solid.shape, np.float32)
    hulls, props = [], []
    Xc = (np.arange(nx) + 0.5) * dx
    if fleet.enabled and fleet.n_boats > 0:
        hulls, props = _place_fleet(fleet, sec, h, cfg, solid, Fx, Fy, Fz, Xc, y, zc, dx, notes)
        notes = list(dict.fromkeys(notes))

    dt = _time_step(cfg, dx, nx, V, uin, props, Fx, Fy, Fz)
    k = dt * dt / (RHO * dx)                     # N/m^3 -> lattice force
    cf, bedwall = wall_cf(solid, bed, dx, sec.n, cfg) if cfg.wall_model else (None, None)
    return Reach(sec=sec, cfg=cfg, fleet=fleet, h=h, Q=Q, S=S, dx=dx, dt=dt, nx=nx, ny=ny, nz=nz, y=y, zc=zc,
                 solid=solid, uin_phys=uin, Fx=(Fx * k).astype(np.float32), Fy=(Fy * k).astype(np.float32),
                 Fz=(Fz * k).astype(np.float32), cf=cf, bedwall=bedwall, hulls=hulls, props=props, notes=notes,
                 W=Wtop, A=A, V=V, body=hull_ids(solid, bed, hulls, Xc, y, zc))


def hull_ids(solid, bed, hulls, Xc, y, zc):
    """The body map of the force readouts: hull k's solid cells (solid, not bed, inside hull k's
    box) hold k + 1, all other cells 0; None without hulls."""
    if not hulls:
        return None
    if len(hulls) > 255:
        raise ValueError("more than 255 hulls")
    hull = solid & ~(bed[:, :, None] if bed.ndim == 2 else bed)
    body = np.zeros(solid.shape, np.uint8)
    for k, (x0, x1, y0, y1, z0, _) in enumerate(hulls):
        box = (zc >= z0)[:, None, None] & ((y >= y0) & (y <= y1))[None, :, None] & ((Xc >= x0) & (Xc <= x1))[None, None, :]
        body[box & hull] = k + 1
    return body


# ------------------------------------------------------------------------------ wall friction
_D3Q19_NEIGHBOURS = np.ones((3, 3, 3), bool)
_D3Q19_NEIGHBOURS[::2, ::2, ::2] = False        # the 18 links of D3Q19 (no cube corners)


def log_cf(z, ks):
    """Rough-wall friction coefficient at distance z (log law, z0 = ks/30): tau = rho cf u^2."""
    return (0.41 / math.log(max(30.0 * z / max(ks, 1e-6), 2.0))) ** 2


def manning_ks(n):
    """Equivalent sand roughness (m) of Manning's n (Strickler)."""
    return (21.1 * n) ** 6


def _touching(mask, solid, floor):
    """Fluid cells linked (D3Q19) to `mask`; `floor` says whether the bed below z=0 and the
    two y edges of the domain count as part of it."""
    pad = np.pad(mask, ((1, 1), (1, 1), (0, 0)), constant_values=False)
    pad[0] = floor
    pad[:, 0] = pad[:, -1] = floor
    pad = np.pad(pad, ((0, 0), (0, 0), (1, 1)), mode="edge")
    return binary_dilation(pad, _D3Q19_NEIGHBOURS)[1:-1, 1:-1, 1:-1] & ~solid


def wall_cf(solid, bed2, dx, n, cfg: ReachConfig):
    """cf of wall-adjacent fluid cells and the bed/bank mask (floodsim/reach3d.py:315-343).

    bed2 is the bed mask: the (nz, ny) section of an extruded reach, or (nz, ny, nx).

    Bed and banks: cf = g n^2 / h_col^(1/3) (h_col = water depth of the column), used with
    the column depth-mean speed.  Hulls: log law from hull_ks with the cell's own speed.
    The first and last two x columns (inlet/outlet) keep plain bounce-back.
    """
    extruded = bed2.ndim == 2                    # (nz, ny) section, or a (nz, ny, nx) bed
    bed = np.broadcast_to(bed2[:, :, None], solid.shape) if extruded else bed2
    hull = solid & ~bed
    cf = np.zeros(solid.shape, np.float32)
    cf[_touching(hull, solid, False)] = log_cf(0.5 * dx, cfg.hull_ks)
    bedwall = _touching(bed, solid, True)
    hcol = np.maximum((~bed2).sum(0) * dx, dx)
    cf_col = (G * n * n / hcol ** (1 / 3)).astype(np.float32)
    cf = np.where(bedwall, cf_col[None, :, None] if extruded else cf_col[None, :, :], cf)
    for a in (cf, bedwall):
        a[:, :, :2] = 0
        a[:, :, -2:] = 0
    return cf.astype(np.float32), bedwall


# ------------------------------------------------------------------------------ time loop
class Run3D:
    """One case on the B200 solver (floodsim/reach3d.py:378-497).

    advance(n) runs n steps in chunks of at most 20: the force ramp is a scalar the kernel
    applies, the bed/bank reference speed is the column mean the kernel refreshes at the
    end of every chunk, and once t >= t_avg the last step of each chunk adds the fields to
    the time-average sums.
    """

    avg_every = 20

    def __init__(self, reach: Reach, be=None, tile=None, storage="fp32", sponge=None):
        self.r, self.be = reach, be
        nu_lb = max(1e-6 * reach.dt / reach.dx ** 2, 2e-4)
        uin_lb = (reach.uin_phys / reach.vel).astype(np.float32)
        column = reach.bedwall is not None
        self.lbm = LBM3D(be, reach.solid, reach.Fx, reach.Fy, reach.Fz, uin_lb, tau0=0.5 + 3 * nu_lb,
                         cs=reach.cfg.cs, cf_wall=reach.cf, bedwall=reach.bedwall,
                         uref_mode="column" if column else "field", tile=tile, storage=storage, sponge=sponge)
        self.xp = self.lbm.xp
        self.lbm.enable_averaging()
        self.navg = 0
        self.t = 0.0
        self.t_total = reach.cfg.run_flows * reach.cfg.length / max(reach.V, 0.05)
        self.t_avg = self.t_total * (1 - reach.cfg.avg_frac)
        self.t_ramp = min(0.15 * self.t_total, 20.0) if reach.props else 0.0
        self._ramp_done = self.t_ramp <= 0
        if not self._ramp_done:
            self.lbm.force_scale = 0.0
        self.steps_wall = 0.0
        self.particles = None
        self._body_dev = None

    @property
    def done(self):
        return self.t >= self.t_total

    def advance(self, nsteps: int):
        t0 = time.time()
        L = self.lbm
        k = 0
        while k < nsteps:
            m = min(self.avg_every, nsteps - k)
            if not self._ramp_done:
                f = min(self.t / self.t_ramp, 1.0)
                f = np.float32(f * f * (3 - 2 * f))
                L.force_scale = float(f)
                self._ramp_done = f >= 1.0
            t_next = self.t + m * self.r.dt
            accumulate = t_next >= self.t_avg
            L.step(m, accumulate=accumulate)
            k += m
            self.t = t_next
            if accumulate:
                self.navg += 1
        self.xp.cuda.synchronize(L.device)
        self.steps_wall += time.time() - t0

    def run_to_end(self, progress=None, cancel=None, chunk=400):
        while not self.done:
            self.advance(chunk)
            if progress:
                progress(self.t / self.t_total)
            if cancel and cancel():
                break

    def mlups(self):
        return self.lbm.nstep * self.r.cells / max(self.steps_wall, 1e-9) / 1e6

    def body_forces(self) -> dict:
        """Float64 force sums on the device, in newtons (x downstream, y across, z up): `hulls`
        (one row per hull of r.hulls, the momentum-exchange force the water exerts on it at the
        current state) and `applied` (the body force of the propellers and jets the step applies,
        the force ramp included).  Needs the reach's hull map (build_reach makes it)."""
        r = self.r
        nb = len(r.hulls)
        if nb and r.body is None:
            raise ValueError("body_forces needs the reach's hull map (Reach.body)")
        if self._body_dev is None and nb:
            self._body_dev = self.lbm._pitched(r.body, self.xp.uint8)
        hulls, applied = self.lbm.body_forces(self._body_dev if nb else None, nb)
        to_n = RHO * r.dx ** 4 / r.dt ** 2
        return {"hulls": hulls * to_n, "applied": applied * to_n}

    def field(self, name: str, mean: bool = False) -> np.ndarray:
        """A field in physical units as a NumPy (nz, ny, nx) array: ux/uy/uz/sp in m/s,
        rho as the equivalent water level (m), uxx in m^2/s^2."""
        L, r = self.lbm, self.r
        if mean and self.navg > 0:
            a = L.avg_sum(name).cpu().numpy() / self.navg
        elif name == "sp":
            a = (L.ux * L.ux + L.uy * L.uy + L.uz * L.uz).sqrt().cpu().numpy()
        elif name == "uxx":
            a = (L.ux * L.ux).cpu().numpy()
        else:
            a = getattr(L, name).cpu().numpy()
        return _physical(r, name, a)

    # ---- tracer particles (floodsim/reach3d.py:499-541), advected on the device
    def init_particles(self, n, seed=None):
        """n particles at uniform positions inside random fluid cells (NumPy generator seeded
        0, as the reference draws them); `seed` seeds the device generator of restarts."""
        import torch
        r = self.r
        rng = np.random.default_rng(0)
        fluid = np.argwhere(~r.solid)
        pick = fluid[rng.integers(0, len(fluid), n)]
        P = (pick[:, ::-1] + rng.random((n, 3))) * r.dx
        dev = self.lbm.device
        self.P = torch.as_tensor(np.ascontiguousarray(P, np.float64), device=dev)
        inlet = np.argwhere(~r.solid[:, :, 1])                      # (z, y) of the x = 1 column's fluid
        self._inlet = torch.as_tensor((inlet[:, 0] * r.ny + inlet[:, 1]).astype(np.int32), device=dev)
        self._respawned = torch.zeros(1, dtype=torch.int32, device=dev)
        self._pseed = int(np.random.SeedSequence(seed).generate_state(1, np.uint64)[0]) if seed is None \
            else int(seed)
        self._pcount = 0
        self.particles = True

    def move_particles(self, dt_phys):
        """One advection step of dt_phys seconds through the current velocity field; particles
        that leave the fluid restart at the inlet (lbm_move_particles)."""
        if not self.particles:
            return
        from . import _native as nat
        from .lbm3d import ctypes_ptr
        import ctypes
        L = self.lbm
        lat = L._lattice()
        self._pcount += 1
        nat.check(L.lib.lbm_move_particles(ctypes.byref(lat), ctypes_ptr(self.P), int(self.P.shape[0]),
                                           float(np.float32(self.r.vel)), float(np.float32(dt_phys)), float(self.r.dx),
                                           ctypes_ptr(self._inlet), int(self._inlet.numel()), self._pseed,
                                           self._pcount, ctypes_ptr(self._respawned), L._stream()),
                  "lbm_move_particles")

    def particles_xyz(self):
        """Positions in metres: x from the inlet, y from the channel centreline, z from the bed
        datum (floodsim/reach3d.py:538-541)."""
        r = self.r
        P = self.P.cpu().numpy()
        return P[:, 0], P[:, 1] + r.y[0] - 0.5 * r.dx, P[:, 2]


# ------------------------------------------------------------------------------ readouts
AVG_KEYS = ("ux", "uy", "uz", "rho", "sp", "uxx")    # the time-average sums of Run3D


def _physical(r: Reach, name: str, a) -> np.ndarray:
    """A lattice-unit field (flat, reference layout) as a (nz, ny, nx) array in physical units,
    as floodsim/reach3d.py:473-486 converts it: rho to the equivalent water level (m), uxx to
    m^2/s^2, velocities and speed to m/s."""
    a = a.reshape(r.nz, r.ny, r.nx)
    if name == "rho":
        return r.eta_from_rho(a)
    if name == "uxx":
        return a * r.vel ** 2
    return a * r.vel


def profiles_from_sums(r: Reach, sums: dict, navg: int) -> dict:
    """profiles() of host time-average sums (float32 arrays in the reference layout, keyed
    ux, uy, uz, rho, sp, uxx) accumulated over `navg` outputs."""
    return _profiles(r, lambda name: _physical(r, name, sums[name] / navg))


def profiles(run: Run3D) -> dict:
    """Along-stream profiles from the time-averaged fields (floodsim/reach3d.py:545-568)."""
    return _profiles(run.r, lambda name: run.field(name, mean=True))


def _profiles(r: Reach, mean_field) -> dict:
    ux = mean_field("ux")
    sp = mean_field("sp")
    eta = mean_field("rho")
    fl = ~r.solid
    top = fl[-1]
    n_top = np.maximum(top.sum(0), 1)
    eta_x = (eta[-1] * top).sum(0) / n_top
    us_x = (ux[-1] * top).sum(0) / n_top
    umax_x = np.where(fl, sp, 0).max(axis=(0, 1))
    q_x = (ux * fl).sum(axis=(0, 1)) * r.dx * r.dx
    uxx = mean_field("uxx")
    mom_x = ((RHO * uxx + RHO * G * eta) * fl).sum(axis=(0, 1)) * r.dx * r.dx
    below = np.concatenate([np.ones((1,) + fl.shape[1:], bool), ~fl[:-1]], 0)
    first = fl & below
    cf = log_cf(0.5 * r.dx, manning_ks(r.sec.n))
    tau = np.where(first, RHO * cf * sp ** 2, 0.0)
    tau_bed = tau.max(axis=0)
    return dict(x=r.x, eta=eta_x - eta_x[-1], us=us_x, umax=umax_x, q=q_x, tau_bed=tau_bed,
                tau_max_x=tau_bed.max(0), mom=mom_x)


def profiles_device(run: Run3D, mean: bool = True) -> dict:
    """profiles() from float64 reductions on the device (lbm_profiles): the same quantities,
    summed in float64 over each cross-section instead of float32 NumPy sums on the host.
    mean=False reads the current (instantaneous) fields."""
    r = run.r
    s = run.lbm.profile_sums(mean=mean)
    vel = r.vel
    n_top = np.maximum(s["top_n"], 1.0)
    eta_x = s["top_drho"] / n_top / 3.0 * vel ** 2 / G
    us_x = s["top_ux"] / n_top * vel
    umax_x = s["umax"] * vel
    q_x = s["q"] * vel * r.dx * r.dx
    mom_x = RHO * vel ** 2 * (s["uxx"] + s["drho"] / 3.0) * r.dx * r.dx
    cf = log_cf(0.5 * r.dx, manning_ks(r.sec.n))
    tau_bed = RHO * cf * s["bed_speed2"] * vel ** 2
    return dict(x=r.x, eta=eta_x - eta_x[-1], us=us_x, umax=umax_x, q=q_x, tau_bed=tau_bed,
                tau_max_x=tau_bed.max(0), mom=mom_x, mass=float(s["mass"].sum()),
                fluid_cells=float(s["n_fluid"].sum()))


def compare(res: dict, base: dict, reach: Reach, cfg: ReachConfig) -> dict:
    """Boat case against the base case (floodsim/reach3d.py:571-618)."""
    x = res["x"]
    fl = reach.fleet
    T, P = fl.total_thrust(), fl.total_power()
    xs = [p["x"] for p in reach.props]
    x_last = max(xs) if xs else 0.0
    i_up = max(int(0.08 * len(x)), 1)
    if reach.hulls:     # the upstream level is read ahead of the first boats
        i_up = max(min(i_up, int(np.searchsorted(x, min(hb[0] for hb in reach.hulls) - 10.0))), 1)
    d_eta = (res["eta"][i_up] - res["eta"][-1]) - (base["eta"][i_up] - base["eta"][-1])
    excess = res["umax"] - base["umax"]
    thr = max(0.2, 0.15 * reach.V)
    down = x > x_last
    hit = np.flatnonzero(down & (excess > thr))
    reach_m = float(x[hit[-1]] - x_last) if len(hit) else 0.0
    reach_capped = bool(len(hit) and hit[-1] >= len(x) - 3)
    m = down & (x < x[-1] - 2 * reach.dx)
    us_gain = float((res["us"][m] - base["us"][m]).mean()) if m.any() else 0.0
    a_cell = reach.dx * reach.dx
    x0 = min([hb[0] for hb in reach.hulls], default=0.15 * x[-1]) - 5.0
    zone = (x >= max(x0, 0.1 * x[-1])) & (x <= x[-1] - 3 * reach.dx)
    tb, tbb = res["tau_bed"][:, zone], base["tau_bed"][:, zone]
    over = float((tb > cfg.tau_crit).sum() * a_cell)
    over_b = float((tbb > cfg.tau_crit).sum() * a_cell)
    i_out = len(x) - 4
    dm = res["mom"] - base["mom"]
    F_net = float(dm[i_out] - dm[i_up])
    gravity = RHO * G * reach.A * cfg.spacing_km * 1000 * max(reach.S, 1e-7)

    def dq(F):
        return math.sqrt(max(1 + F / gravity, 0.0)) - 1

    dQ, dQn = dq(T), dq(F_net)
    return dict(label=fl.label(), n=fl.n_boats, T_kN=T / 1000, P_kW=P, h=reach.h, Q=reach.Q, V=reach.V,
                d_eta_cm=100 * d_eta, jet_reach=reach_m, reach_capped=reach_capped,
                us_gain=us_gain, us_gain_pct=100 * us_gain / max(reach.V, 1e-6),
                umax=float(res["umax"].max()), tau_max=float(tb.max()), tau_base=float(tbb.max()),
                tau_area=over, tau_area_base=over_b, dQ_pct=100 * dQ, dQ_net_pct=100 * dQn,
                F_net_kN=F_net / 1000, dQ_per_100kW=100 * dQn / max(P / 100, 1e-9) if P > 0 else 0.0,
                drop_cm_per_100kW=-100 * d_eta / (P / 100) if P > 0 else 0.0,
                kW_per_cm=P / (-100 * d_eta) if (P > 0 and d_eta < -1e-5) else float("nan"),
                T_per_kW=T / max(P, 1e-9) if P > 0 else 0.0)
