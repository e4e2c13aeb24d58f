"""The C-ABI library: it builds for sm_100a, loads without a GPU, exports every
function include/lbm_b200.h declares, and its structs match the header layout."""
import ctypes
import os
import re
import subprocess

import pytest

from water_flow_simulation_b200 import _native as nat

HEADER = os.path.join(nat.INCLUDE, "lbm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(lbm_\w+)\s*\(", src, flags=re.M)))


def test_library_builds_and_loads():
    lib = nat.load()
    assert lib.lbm_abi_version() == nat.ABI_VERSION
    m = re.search(r"#define LBM_ABI_VERSION (\d+)", open(HEADER).read())
    assert m and int(m.group(1)) == nat.ABI_VERSION
    assert lib.lbm_last_error() == b""


def test_every_declared_symbol_is_exported_and_bound():
    lib = nat.load()
    names = declared_functions()
    assert {"lbm_step", "lbm_bc", "lbm_fused_step", "lbm_build_flags", "lbm_init_equilibrium"} <= set(names)
    for n in names:
        assert hasattr(lib, n), n
        assert n in nat.SIGNATURES, f"{n} has no ctypes signature"


def test_struct_layout_matches_header(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "lbm_b200.h"\n'
                    'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(lbm_lattice), '
                    'offsetof(lbm_lattice, flags), offsetof(lbm_lattice, status), sizeof(lbm_tile), '
                    'offsetof(lbm_lattice, cells));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", nat.INCLUDE, "-o", str(exe), str(prog)])
    got = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    L = nat.Lattice
    assert got == [ctypes.sizeof(L), L.flags.offset, L.status.offset, ctypes.sizeof(nat.Tile), L.cells.offset]


def test_argument_errors_are_status_codes_not_crashes():
    """Bad arguments are rejected on the host before any launch (no GPU needed)."""
    lib = nat.load()
    assert lib.lbm_step(None, None, None, None, None, None, None, None, None, None, None, None,
                        8, 8, 8, 0.6, 0.03, None) == -1
    assert b"NULL" in lib.lbm_last_error()
    L = nat.Lattice()
    L.nx, L.ny, L.nz, L.pitch, L.cells = 10, 4, 4, 10, 160
    assert lib.lbm_fused_step(ctypes.byref(L), None, None, 1, None, None) == -1
    assert b"pitch" in lib.lbm_last_error()
    L.pitch, L.cells = 12, 12 * 16
    tile = nat.Tile(3, 4, 0)
    assert lib.lbm_fused_step(ctypes.byref(L), None, None, 1, ctypes.byref(tile), None) == -1


def test_fp64_solver_argument_errors():
    lib = nat.load()
    assert lib.lbm_step_f64(*([None] * 12), 8, 8, 8, 0.6, 0.03, 0, 0.0, None) == -1
    assert b"lbm_step_f64: NULL" in lib.lbm_last_error()
    assert lib.lbm_bc_f64(None, None, None, 8, 8, 8, 1.0, None) == -1
    buf = ctypes.c_double()
    p = ctypes.addressof(buf)
    assert lib.lbm_bc_f64(p, p, p, 2, 8, 8, 1.0, None) == -1
    assert b"bad lattice" in lib.lbm_last_error()
    assert lib.lbm_update_uref_f64(None, None, None, None, None, 8, 8, 8, None) == -1
    assert lib.lbm_step_f64(*([p] * 12), 8, 8, 8, 0.6, 0.03, 0, 0.0, None) == -1      # fs == fd
    assert b"differ" in lib.lbm_last_error()


def test_export_argument_errors():
    lib = nat.load()
    L = nat.Lattice()
    L.nx, L.ny, L.nz, L.pitch, L.cells = 1, 4, 4, 4, 64
    assert lib.lbm_export_blocks(ctypes.byref(L)) == -1
    L.nx, L.ny, L.nz, L.pitch, L.cells = 9, 5, 3, 12, 12 * 15
    assert lib.lbm_export_blocks(ctypes.byref(L)) == 4 * 2 * 3
    assert lib.lbm_export_velocity(ctypes.byref(L), 3, 1.0, None, None, None, None, None) == -1
    assert b"no time averages" in lib.lbm_last_error()


def test_particle_argument_errors():
    lib = nat.load()
    L = nat.Lattice()
    L.nx, L.ny, L.nz, L.pitch, L.cells = 8, 4, 4, 8, 128
    assert lib.lbm_move_particles(ctypes.byref(L), None, 0, 1.0, 1.0, 0.1, None, 0, 1, 1, None, None) == 0
    assert lib.lbm_move_particles(ctypes.byref(L), None, 5, 1.0, 1.0, 0.1, None, 0, 1, 1, None, None) == -1
    assert b"NULL" in lib.lbm_last_error()
    assert lib.lbm_move_particles(None, None, 5, 1.0, 1.0, 0.1, None, 0, 1, 1, None, None) == -1


def test_sponge_argument_errors():
    """The outlet sponge is validated with the lattice (no GPU needed: no launch happens)."""
    import numpy as np
    lib = nat.load()
    buf = np.zeros(4096, np.float32)
    p = buf.ctypes.data
    L = nat.Lattice()
    L.nx, L.ny, L.nz, L.pitch, L.cells = 12, 4, 4, 12, 12 * 16
    L.tau0, L.csmag2 = 0.6, 0.03
    L.flags = L.uin = p
    L.sponge_cols, L.sponge_tau = 11, 0.7                 # more than nx - 2 columns
    assert lib.lbm_init_equilibrium(ctypes.byref(L), p, None) == -1
    assert b"sponge_cols" in lib.lbm_last_error()
    L.sponge_cols, L.sponge_tau = 4, 0.5                  # below tau0
    assert lib.lbm_init_equilibrium(ctypes.byref(L), p, None) == -1
    assert b"sponge_tau" in lib.lbm_last_error()
    L.sponge_tau = 0.7
    L.Fx = L.Fy = L.Fz = L.cfw = L.uref = L.rho = L.ux = L.uy = L.uz = L.status = p
    tile = nat.Tile(1, 1, 4, 4, 0)                        # TMA pipeline
    assert lib.lbm_fused_step(ctypes.byref(L), p, p + 1024, 0, ctypes.byref(tile), None) == -1
    assert b"split pipeline" in lib.lbm_last_error()


def test_16bit_storage_argument_errors():
    """16-bit entry points: the scale must be a power of two, the pitch a multiple of 8, the tile the
    8-cells-per-lane split pipeline; all rejected on the host (no GPU needed)."""
    lib = nat.load()
    dummy = (ctypes.c_uint32 * 64)()
    L = nat.Lattice()
    L.nx, L.ny, L.nz, L.pitch, L.cells = 10, 4, 4, 12, 12 * 16
    L.flags = L.uin = ctypes.addressof(dummy)
    for bad in (0.0, -4.0, 3000.0, 2.0 ** 30, float("nan")):
        assert lib.lbm_init_equilibrium_h(ctypes.byref(L), ctypes.addressof(dummy), bad, None) == -1
        assert b"power of two" in lib.lbm_last_error()
        assert lib.lbm_fused_step_h(ctypes.byref(L), None, None, bad, 1, None, None) == -1
    assert lib.lbm_fused_step_h(ctypes.byref(L), None, None, 2.0 ** 14, 1, None, None) == -1
    assert b"multiple of 8" in lib.lbm_last_error()
    L.pitch, L.cells = 16, 16 * 16
    fake = ctypes.addressof(dummy)
    for k in ("Fx", "Fy", "Fz", "cfw", "uref", "rho", "ux", "uy", "uz", "status"):
        setattr(L, k, fake)
    tile = nat.Tile(3, 3, 4, 0, 0)
    assert lib.lbm_fused_step_h(ctypes.byref(L), fake, fake + 1024, 2.0 ** 14, 1, ctypes.byref(tile), None) == -1
    assert b"2, 4 or 8 cells per lane" in lib.lbm_last_error()
    tile = nat.Tile(3, 8, 4, 0, 0)
    L.list_cells_per_lane = 4
    assert lib.lbm_fused_step_h(ctypes.byref(L), fake, fake + 1024, 2.0 ** 14, 1, ctypes.byref(tile), None) == -1
    assert b"work lists" in lib.lbm_last_error()


def test_solver_refuses_to_run_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import numpy as np
    from water_flow_simulation_b200.lbm3d import LBM3D
    z = np.zeros((4, 4, 8), np.float32)
    with pytest.raises(nat.LBMError):
        LBM3D(None, z.astype(bool), z, z, z, np.zeros((4, 4), np.float32), 0.6)


def test_body_forces_argument_errors():
    """Body-force sums reject a body count over 16 and NULL arrays before any launch."""
    lib = nat.load()
    assert lib.lbm_body_forces_scratch_doubles(17) == -1
    assert b"nbody 17" in lib.lbm_last_error()
    assert lib.lbm_body_forces_scratch_doubles(2) == 1024 * 9
    flags = ctypes.c_uint32()
    L = nat.Lattice()
    L.nx, L.ny, L.nz, L.pitch, L.cells = 8, 4, 4, 8, 128
    L.flags = L.uin = ctypes.addressof(flags)
    assert lib.lbm_body_forces(ctypes.byref(L), None, None, 0, 0, None, None, None) == -1
    assert b"NULL array" in lib.lbm_last_error()
    assert lib.lbm_body_forces_h(ctypes.byref(L), None, 3.0, None, 0, 0, None, None, None) == -1
    assert b"power of two" in lib.lbm_last_error()
