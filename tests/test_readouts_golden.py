"""Host readouts against the reference's own profiles and compare (golden fixtures).

tests/golden/make_golden.py seeds the time-average sums of a reference Run3D for a boat
case and for its no-boat base case, runs the reference's ``profiles`` on both and
``compare`` on the pair (floodsim/reach3d.py:545-618), and stores sums and results.
Here the same sums go through ``reach3d.profiles_from_sums`` (the code ``profiles`` runs
on a finished run's averages) and ``reach3d.compare``: every profile array must be equal
to the reference's bit for bit (the same NumPy operations in the same dtypes), and every
scalar of ``compare`` within 1e-12 relative.
"""
import json
import math
import os

import numpy as np
import pytest

from golden_io import GOLDEN
from test_reach_builder import build_from_spec
from water_flow_simulation_b200.reach3d import AVG_KEYS, compare, profiles_from_sums

CASES = ("mini_tug", "mini_cfg1")
PROFILE_KEYS = ("x", "eta", "us", "umax", "q", "tau_bed", "tau_max_x", "mom")


def _load(name):
    d = np.load(os.path.join(GOLDEN, f"readouts_{name}.npz"))
    spec, base_spec = json.loads(str(d["spec"])), json.loads(str(d["base_spec"]))
    return d, build_from_spec(spec), build_from_spec(base_spec)


def _sums(d, tag):
    return {k: d[f"{tag}_sum_{k}"] for k in AVG_KEYS}, int(d[f"{tag}_navg"])


@pytest.mark.parametrize("name", CASES)
def test_profiles_equal_reference(name):
    d, r, rb = _load(name)
    for tag, reach in (("boat", r), ("base", rb)):
        res = profiles_from_sums(reach, *_sums(d, tag))
        assert set(PROFILE_KEYS) <= set(res)
        for k in PROFILE_KEYS:
            want = d[f"{tag}_res_{k}"]
            got = np.asarray(res[k])
            assert got.shape == want.shape, (tag, k)
            assert got.dtype == want.dtype, (tag, k, got.dtype, want.dtype)
            np.testing.assert_array_equal(got, want, err_msg=f"{name} {tag} {k}")


@pytest.mark.parametrize("name", CASES)
def test_compare_equals_reference(name):
    d, r, rb = _load(name)
    res = profiles_from_sums(r, *_sums(d, "boat"))
    base = profiles_from_sums(rb, *_sums(d, "base"))
    got = compare(res, base, r, r.cfg)
    want = json.loads(str(d["compare"]))
    assert set(want) == set(got)
    for k, v in want.items():
        if k == "label":              # the fleet label is display text (the reference's is Thai)
            continue
        g = got[k]
        if v is None:                 # NaN in the reference (kW_per_cm without a level drop)
            assert isinstance(g, float) and math.isnan(g), (k, g)
        elif isinstance(v, bool):
            assert g == v, (k, g, v)
        else:
            assert abs(g - v) <= 1e-12 * max(abs(v), 1e-30), (k, g, v)
