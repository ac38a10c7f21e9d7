"""Times the 64-case 200 MiB sweep under several per-case schedule rules, on one GPU.

    python -m ttc_b200.sweep_schedules --preset PRESET [--repeats 2] [--seed 2024]

PRESET: bulk, tile_order, lane_maps, shifted_runs or ring_depth (see PRESETS).

The sweep is the benchmark's (`ttc_b200.workloads.sweep_cases`: seeded rank-2..6 fp32/fp64
transpositions, |A| ~ 200 MiB, half with alpha = 1.5, beta = -0.5). Inputs are seeded on the device
once. For each repeat and each rule of the preset, one plan is made per case with the schedule the
rule gives it; then the sweep is run twice untimed, four times back to back between two CUDA events
(the total), and three times with events around every call (the per-case figures, medians). The
rules run in turn within each repeat, so that drift on the box reaches all of them alike.

One JSON line per (repeat, rule): the total GB/s (algorithmic bytes over the back-to-back time),
the per-case GB/s, the number of bulk-copy stage waits that ran out of time, and per case the bytes
that one bulk copy moves under that rule (0 where the plan has no bulk copies).
"""
from __future__ import annotations

import argparse
import json
import math
import statistics
from typing import Callable, Optional

from .autotune import ELEM_BYTES
from .core import plan_host_json, split_dtype

BULK_MIN_BYTES = 320  # bulk copies of fewer bytes measured slower than per-thread copies


def bulk_copy_bytes(desc: dict, dtype: str) -> int:
    """Bytes one bulk copy moves in a plan (the A run, or its piece when the staged layout's padding
    period cuts it); 0 when the plan makes no bulk copies."""
    t = desc.get("tile") or {}
    if desc.get("kernel") != "tile" or not t.get("bulk"):
        return 0
    ea = ELEM_BYTES[split_dtype(dtype)[0]]
    run = t["LA"]
    sigma = t.get("sigmaA") or run
    if not t.get("shifted_runs") and sigma < run:
        run = sigma
    return int(run * ea)


def _bulk_if_long(base: dict) -> Callable[[dict], Optional[dict]]:
    """The schedule `base` plus bulk copies, where the bulk plan's copies are BULK_MIN_BYTES or more."""
    def rule(c: dict) -> Optional[dict]:
        tu = dict(base, bulk_copies=1)
        d = plan_host_json(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning=tu)
        return tu if bulk_copy_bytes(d, c["dtype"]) >= BULK_MIN_BYTES else (dict(base) or None)
    return rule


def _fixed(tu: dict) -> Callable[[dict], Optional[dict]]:
    return lambda c: dict(tu) or None


PRESETS = {
    # how the staged kernel fills a stage with A: per-thread cp.async against cp.async.bulk per run,
    # under each tile order (the planner's claims rule, claimed everywhere, round robin everywhere)
    "bulk": {
        "default": _fixed({}),
        "bulk": _fixed({"bulk_copies": 1}),
        "bulk_320": _bulk_if_long({}),
        "bulk_shifted": _fixed({"bulk_copies": 1, "shifted_runs": 1}),
        "claims": _fixed({"round_robin": -1}),
        "claims_bulk_320": _bulk_if_long({"round_robin": -1}),
        "round_robin": _fixed({"round_robin": 1}),
        "round_robin_bulk": _fixed({"round_robin": 1, "bulk_copies": 1}),
        "round_robin_bulk_320": _bulk_if_long({"round_robin": 1}),
    },
    # the staged kernel's tile order: the planner's claims rule with 1, 2 (its default), 3 or 4 tiles
    # per claim, claims for every tile plan, round robin everywhere
    "tile_order": {
        "default": _fixed({}),
        "group_1": _fixed({"claim_group": 1}),
        "group_3": _fixed({"claim_group": 3}),
        "group_4": _fixed({"claim_group": 4}),
        "claims": _fixed({"round_robin": -1}),
        "claims_group_4": _fixed({"round_robin": -1, "claim_group": 4}),
        "round_robin": _fixed({"round_robin": 1}),
    },
    # the register path's lane maps (a warp's B vectors taken from several B runs)
    "lane_maps": {
        "default": _fixed({}),
        "lane_map": _fixed({"lane_map": 1}),
    },
    # A runs that 16-byte copies cannot reach, copied as the 16-byte chunks that cover them
    "shifted_runs": {
        "default": _fixed({}),
        "shifted_runs": _fixed({"shifted_runs": 1}),
    },
    # the ring depth: the planner's rule (tiles in motion nearest 18 MiB) against fixed depths
    "ring_depth": {
        "default": _fixed({}),
        "stages_3": _fixed({"stages": 3}),
        "stages_4": _fixed({"stages": 4}),
        "stages_5": _fixed({"stages": 5}),
        "stages_6": _fixed({"stages": 6}),
    },
}


def run(preset: str, repeats: int = 2, seed: int = 2024, log=print) -> list[dict]:
    import torch
    from . import workloads as wl
    from .core import Plan
    rules = PRESETS[preset]
    cases = wl.sweep_cases(seed)
    tmap = {"s": torch.float32, "d": torch.float64}
    gen = torch.Generator(device="cuda")
    data = []
    for c in cases:
        n = math.prod(c["size"])
        gen.manual_seed(c["seed"])
        A = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen).mul_(2).sub_(1)
        gen.manual_seed(c["seed"] + 1)
        B = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen).mul_(2).sub_(1)
        data.append((c, A, B))
    schedules = {name: [rule(c) for c in cases] for name, rule in rules.items()}
    st = torch.cuda.current_stream()
    out = []
    for rep in range(repeats):
        for name in rules:
            plans = [Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning=tu)
                     for (c, _, _), tu in zip(data, schedules[name])]

            def sweep(evs=None):
                for k, ((c, A, B), p) in enumerate(zip(data, plans)):
                    if evs:
                        evs[k][0].record(st)
                    p(A, B, c["alpha"], c["beta"], st)
                    if evs:
                        evs[k][1].record(st)
            for _ in range(2):
                sweep()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for _ in range(4):
                sweep()
            e1.record(st)
            torch.cuda.synchronize()
            total_ms = e0.elapsed_time(e1) / 4
            per = [[] for _ in data]
            for _ in range(3):
                evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in data]
                sweep(evs)
                torch.cuda.synchronize()
                for k, (a, b) in enumerate(evs):
                    per[k].append(a.elapsed_time(b))
            nbytes = sum(p.bytes for p in plans)
            row = {"repeat": rep, "rule": name, "total_GBps": round(nbytes / total_ms / 1e6, 1),
                   "per_case_GBps": [round(p.bytes / statistics.median(m) / 1e6, 1) for p, m in zip(plans, per)],
                   "wait_timeouts": sum(p.wait_timeouts() for p in plans),
                   "bulk_bytes": [bulk_copy_bytes(p.describe(), c["dtype"]) for (c, _, _), p in zip(data, plans)]}
            for p in plans:
                p.close()
            out.append(row)
            if log:
                log(json.dumps(row))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--preset", default="bulk", choices=sorted(PRESETS))
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args(argv)
    run(a.preset, a.repeats, a.seed)


if __name__ == "__main__":
    main()
