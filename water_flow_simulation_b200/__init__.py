"""B200-native D3Q19 lattice-Boltzmann hot path of floodsim (ThTpk/water_flow_simulation).

``LBM3D`` is the drop-in solver object behind the reference's solver API
(floodsim/lbm3d.py); the kernels live in liblbm_b200.so (csrc/, C ABI in
include/lbm_b200.h).
"""
from .lbm3d import LBM3D  # noqa: F401

__all__ = ["LBM3D"]
