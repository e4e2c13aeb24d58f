"""The kernels' wall function (d3q19.cuh) against the reference's per-direction form, on the CPU.

tests/native/wall_function_check.cu compiles d3q19.cuh as host code (nvcc, no GPU needed) and
runs both forms on 200,000 random wall masks, populations and previous-step velocities: the
regrouped float64 sums (no unit vectors, two square roots and two divisions) must give every
updated population to within float32 rounding of the reference form (floodsim/lbm3d.py:224-252),
i.e. at most one float32 unit in the last place apart.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc (host compilation only)")
def test_wall_function_matches_reference_form(tmp_path):
    exe = tmp_path / "wfc"
    subprocess.check_call(["nvcc", "-O2", "-std=c++17", "-x", "cu", os.path.join(HERE, "native", "wall_function_check.cu"),
                           "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    updated, cases, changed, worst = int(out[0]), int(out[1]), int(out[2]), float(out[3])
    assert cases == 200000 and updated > 100000      # most random masks give a usable wall normal
    assert worst <= 2.0 ** -23, (changed, worst)
