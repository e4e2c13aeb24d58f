"""bench.py's host-side pieces that need no GPU: the accuracy block it reports beside the
bench line, read from the committed statement of the benchmark case."""
import json
import os

import bench


def test_accuracy_block_reads_the_committed_statement():
    """level_error_vs_fp64 carries, per storage and for the float64 floor, the numbers of
    profiles/accuracy_statement_reach36m.json: level, level-change error, shear (largest and
    bed-averaged) and the discharge-gain error of compare's momentum balance."""
    out = bench.accuracy_statement()
    assert out is not None
    with open(os.path.join(bench.ROOT, "profiles", "accuracy_statement_reach36m.json")) as fh:
        d = json.load(fh)
    assert out["steps"] == d["steps"] and out["averaged_from_step"] == d["avg_from"]
    assert out["fp64_level_change_cm"] == d["level_change"]["fp64"]["d_eta_cm"]
    assert out["fp64_discharge_gain_pct"] == d["boat_effects"]["fp64"]["dQ_net_pct"]
    for k, name in (("fp64p", "fp64_floor"), ("fp32", "fp32"), ("fp16", "fp16")):
        row = out[name]
        assert row["level_max_cm"] == d["boat"][k]["level_max_cm"]
        assert row["level_change_error_cm"] == d["level_change"][k]["error_cm"]
        assert row["shear_avg_rel"] == d["boat"][k]["shear_avg_rel"]
        assert row["discharge_gain_error_pct"] == d["boat_effects"][k]["error"]["dQ_net_pct"]
    # the statement the metric rests on: the 16-bit store within 0.5 cm of float64 in level
    assert out["fp16"]["level_max_cm"] < 0.5 and abs(out["fp16"]["level_change_error_cm"]) < 0.5
