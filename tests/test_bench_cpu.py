"""Host-side helpers of the benchmark and the launch accounting (no GPU)."""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def test_parse_cpulist():
    import bench
    assert bench.parse_cpulist("0-3,8,10-11\n") == {0, 1, 2, 3, 8, 10, 11}
    assert bench.parse_cpulist("5") == {5}
    assert bench.parse_cpulist("") == set()


def test_describe_launches_counts_edge_plans():
    """A call launches the plan's kernel, and for a staged tile plan with ragged tiles its edge plans'
    kernels (each with its own ragged-tile kernel when it has ragged tiles) or, without edge plans,
    the element-wise ragged-tile kernel."""
    from ttc_b200.core import describe_launches
    row = {"kernel": "row"}
    plain = {"kernel": "tile", "tile": {"async": 1, "ragged_tiles": 0}}
    edge_ragged = {"kernel": "tile", "tile": {"async": 1, "ragged_tiles": 3}}
    assert describe_launches(row) == 1
    assert describe_launches(plain) == 1
    assert describe_launches(edge_ragged) == 2  # no edge plans: the ragged-tile kernel
    parent = {"kernel": "tile", "tile": {"async": 1, "ragged_tiles": 9},
              "edges": [{"offA": 0, "offB": 0, "plan": plain}, {"offA": 5, "offB": 7, "plan": edge_ragged}]}
    assert describe_launches(parent) == 1 + 1 + 2
    legacy = dict(parent, tile_variant=1)  # the legacy kernels move ragged tiles inline
    assert describe_launches(legacy) == 1


def test_knob_counts_and_schedule_kinds():
    """The sweep line's `schedule_kinds` counts, per kind of schedule, the cases whose schedule sets
    each tuning field (copy form and tile order with their values), and every kind has its note."""
    import bench
    tunings = [None, {"bulk_copies": 1, "stages": 4}, {"round_robin": -1, "stages": 5},
               {"shifted_runs": 1, "bulk_copies": 1}, {}]
    assert bench.knob_counts(tunings) == {"bulk_copies=1": 2, "round_robin=-1": 1, "shifted_runs=1": 1,
                                          "stages": 2}
    assert bench.knob_counts([None, {}]) == {}
    import numpy as np
    assert bench.plain_json({"stages": np.int64(4), "raster": [np.int32(2), 1]}) == {"stages": 4, "raster": [2, 1]}
    args = bench.parse([])
    assert args.schedule == "search" and args.search_candidates == 200
    assert set(bench.SCHEDULE_NOTES) == {"search", "learned", "default"}
    assert bench.parse(["--schedule", "learned"]).schedule == "learned"


def test_sweep_schedule_rules():
    """The schedule-comparison presets (host planning only): bulk copies are asked for only where
    the planner can make them, the bytes per bulk copy follow the staged layout's pieces, and the
    320-byte rule keeps the long copies."""
    from ttc_b200 import sweep_schedules as ss
    from ttc_b200.core import plan_host_json
    from ttc_b200.workloads import sweep_cases
    cases = sweep_cases(2024)
    rules = ss.PRESETS["bulk"]
    assert rules["default"](cases[0]) is None
    assert ss.PRESETS["tile_order"]["group_3"](cases[0]) == {"claim_group": 3}
    assert ss.PRESETS["lane_maps"]["lane_map"](cases[0]) == {"lane_map": 1}
    assert rules["round_robin"](cases[0]) == {"round_robin": 1}
    for c in cases:
        d = plan_host_json(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning={"bulk_copies": 1})
        nb = ss.bulk_copy_bytes(d, c["dtype"])
        assert nb == 0 or nb % 16 == 0, (c, nb)  # whole 16-byte vectors
        long_rule = rules["bulk_320"](c)
        assert (long_rule == {"bulk_copies": 1}) == (nb >= ss.BULK_MIN_BYTES), (c, nb, long_rule)
    # sweep case 25 (fp64, runs of 96 elements, one bulk copy per run) and case 6 (fp64, 1920-element
    # runs cut into 40-element pieces at the padding points)
    for k, want in ((25, 768), (6, 320)):
        c = cases[k]
        d = plan_host_json(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning={"bulk_copies": 1})
        assert ss.bulk_copy_bytes(d, c["dtype"]) == want
