"""Measured search over the schedule space, the counterpart of TTC's exhaustive variant timing
(ttc.py:847-1022, GPUtransposeGenerator.py:165-230 in the TTC project).

TTC generates every (blocking x loop order) variant as source, compiles them all and times each
with wall-clock around the wrapper. Here a candidate is a `ttcb_tuning` (tile size target, run
length target, tile kernel variant, grid raster order, CTA count): the planner turns it into a plan
in microseconds, so the search costs only kernel time. Candidates are deduplicated by the plan they
produce, ordered by the planner's cost estimate and capped at maxImplementations, like TTC's
pruning. Every candidate's output is compared with the first candidate's (all schedules must agree
bit for bit); timing uses CUDA events around each launch with the L2 flushed in between, minimum
over repetitions.
"""
from __future__ import annotations

import itertools
import math
import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

from .core import ELEM_BYTES, Plan, plan_shapes, split_dtype

SMS = 148
L2_BYTES = 126 * 1024 * 1024


class L2Flush:
    """Evicts the L2 between timed launches: writes a buffer twice the L2's size, then reads another
    one as large. The reads push the written lines back to HBM before the next launch, so that launch
    starts with an L2 of clean lines that hold none of its data and pays for no write-back of the
    flush itself (a flush by writing alone leaves up to the L2's size of dirty lines, whose write-back
    would be charged to the kernel timed next)."""

    def __init__(self, device="cuda"):
        import torch
        self.w = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=device)
        self.r = torch.zeros(2 * L2_BYTES // 4, dtype=torch.float32, device=device)
        self.out = torch.empty((), dtype=torch.float32, device=device)

    def __call__(self):
        import torch
        self.w.zero_()
        torch.sum(self.r, dim=0, out=self.out)


@dataclass
class Problem:
    perm: list
    size: list
    dtype: str = "s"
    alpha: complex | float = 1.0
    beta: complex | float = 0.0
    lda: Optional[list] = None
    ldb: Optional[list] = None

    @property
    def beta_nonzero(self) -> bool:
        return complex(self.beta) != 0

    def elements(self) -> int:
        return math.prod(self.size)

    def bytes(self) -> int:
        ta, tb = split_dtype(self.dtype)
        return self.elements() * (ELEM_BYTES[ta] + ELEM_BYTES[tb] * (2 if self.beta_nonzero else 1))

    def buffer_elems(self):
        la = self.lda or self.size
        lb = self.ldb or [self.size[p] for p in self.perm]
        na = math.prod(la[:-1]) * self.size[-1]
        nb = math.prod(lb[:-1]) * self.size[self.perm[-1]]
        return max(na, 1), max(nb, 1)


@dataclass
class Result:
    tuning: dict
    time_ms: float
    gbs: float
    desc: dict = field(default_factory=dict)
    ok: bool = True


def knob_space(dtype: str, ttc_orders: int = 0) -> dict:
    """The schedule knobs the search crosses. `ttc_orders` > 0 adds, per tile shape, up to that many
    explicit loop orders from TTC's own ranking (see ranked_loop_orders) whose raster differs from
    the preset orders'."""
    ta, _ = split_dtype(dtype)
    base = 16384 // ELEM_BYTES[ta]
    return {
        "rasters": ("ttc", ttc_orders) if ttc_orders else [],
        "tile_elems": [0, base // 4, base // 2, base * 2],
        "run_bytes": [0, 128, 256, 512, 1024, 2048],
        # the register-prefetch (2) and table-driven (1) tile kernels were the fastest schedule for 12
        # of the 2000 timed training problems (none by more than noise on the 500 held out) while
        # taking a fifth of the candidates, so the search leaves them to explicit schedules
        "tile_variant": [0],
        "loop_order": [0, 1, 2, 3],
        "blocks": [0],
        # the staged kernel's ring depth x CTAs per SM besides the planner's: the `schedules` pairs
        # whose tiles in motion come closest to the planner's target (see schedule_alternatives)
        "schedules": 3,
    }


TARGET_IN_FLIGHT = 18 * 1024 * 1024  # the planner's target for the bytes of tiles in motion


def schedule_alternatives(p: Problem, desc: dict, k: int) -> list[dict]:
    """Up to k (stages, ctas_per_sm) pairs other than the planner's own for a staged-kernel tile,
    nearest the planner's in-flight target first (W = CTAs x (stages - 1) x tile bytes), skipping
    rings that would not fit the kernel's shared memory; then tiles claimed in order from counters,
    bulk A copies where 16-byte vectors reach A's runs, and otherwise shifted A runs (with per-thread
    or bulk copies) where the runs are long enough."""
    t = desc.get("tile") or {}
    if desc["kernel"] != "tile" or k <= 0 or not t.get("P"):
        return []
    ta, tb = split_dtype(p.dtype)
    ea, eb = ELEM_BYTES[ta], ELEM_BYTES[tb]
    P = t["P"]
    tile_bytes = P * (ea + eb * (2 if p.beta_nonzero else 1))
    stage = P * ea * 1.07 + (P * eb if p.beta_nonzero else 0)
    cmax = lambda S: max(1, min(4, int(227 * 1024 // (S * stage + 3 * 1024))))
    mine = (t.get("stages"), t.get("ctas_per_sm") or cmax(t.get("stages") or 3))
    opts = []
    for S in (3, 4, 5, 6):
        if S * stage > 200 * 1024:
            continue
        for c in (2, 3, 4):
            if c > cmax(S) or (S, c) == mine:
                continue
            W = c * SMS * (S - 1) * tile_bytes
            # fewer CTAs than fit cost the sweep 2-12%, so they come after every full-occupancy ring
            opts.append((c != cmax(S), abs(math.log(W / TARGET_IN_FLIGHT)), c, S))
    out = [{"stages": S, "ctas_per_sm": c} for _, _, c, S in sorted(opts)[:k]]
    # the other tile order and the other way of moving A than the planner's
    out.append({"round_robin": 1 if staged_claims(p, {}, desc) else -1})
    vm = 16 // ea
    if desc.get("vecA", vm) * ea == 16:
        out.append({"bulk_copies": 1})
    elif t.get("LA", 0) >= 2 * vm:
        # A runs that 16-byte copies cannot reach directly, copied as covering 16-byte chunks
        out += [{"shifted_runs": 1}, {"shifted_runs": 1, "bulk_copies": 1}]
    return out


def staged_claims(p: Problem, tuning: dict, desc: dict) -> bool:
    """Whether the staged kernel claims tiles from counters under this schedule: asked for
    (round_robin -1), or the planner's rule for round_robin 0 - tiles of 16 KiB or more (A, B and B
    read back) with 16 or more per CTA (CTAs estimated as SMs x the schedule's CTAs per SM, else as
    many as the ring's shared memory lets share an SM)."""
    rr = tuning.get("round_robin", 0)
    if rr != 0:
        return rr == -1
    t = desc.get("tile") or {}
    if desc.get("kernel") != "tile" or not t.get("P"):
        return False
    ta, tb = split_dtype(p.dtype)
    tile_bytes = t["P"] * (ELEM_BYTES[ta] + ELEM_BYTES[tb] * (2 if p.beta_nonzero else 1))
    c = tuning.get("ctas_per_sm") or t.get("ctas_per_sm") or 0
    if not c:
        stage = t["P"] * ELEM_BYTES[ta] * 1.07 + (t["P"] * ELEM_BYTES[tb] if p.beta_nonzero else 0)
        S = tuning.get("stages") or t.get("stages") or 3
        c = max(1, min(4, int(227 * 1024 // (S * stage + 3 * 1024))))
    ctas = tuning.get("blocks") or c * SMS
    return tile_bytes >= 16 * 1024 and t.get("ntiles", 0) >= 16 * ctas


def fused_groups(p: Problem):
    """The library's index fusion of a problem (host only): (fused perm, fused sizes, groups), where
    groups[i] lists the caller's dimensions of fused dimension i in A order; extent-1 dimensions are
    in no group."""
    from .core import fuse
    la = p.lda or p.size
    lb = p.ldb or [p.size[q] for q in p.perm]
    r = len(p.size)
    sA, sBp = [1] * r, [1] * r
    for i in range(1, r):
        sA[i] = sA[i - 1] * la[i - 1]
        sBp[i] = sBp[i - 1] * lb[i - 1]
    sB = [0] * r
    for j, q in enumerate(p.perm):
        sB[q] = sBp[j]
    fperm, fsize, _, _ = fuse(p.perm, p.size, sA, sB)
    groups, cur = [], []
    dims = [d for d in range(r) if p.size[d] != 1]
    k = 0
    for fs in fsize:
        prod, cur = 1, []
        while k < len(dims) and prod < fs:
            prod *= p.size[dims[k]]
            cur.append(dims[k])
            k += 1
        groups.append(cur)
    return fperm, fsize, groups


def ranked_loop_orders(p: Problem, limit: int) -> list[list[int]]:
    """TTC's loop-order heuristic: every order of the fused dimensions ranked by
    ttc_util.getCostLoop, cheapest first, the first `limit` kept (GPUtransposeGenerator.py:203-230,
    ttc_util.py:167-209), each written as an order of the caller's dimensions (extent-1 dimensions
    last) for ttcb_tuning's explicit raster. Fused problems beyond rank 7 are not enumerated."""
    from .ttc_util import getCostLoop
    fperm, fsize, groups = fused_groups(p)
    if len(fsize) > 7 or limit <= 0:
        return []
    ranked = sorted(itertools.permutations(range(len(fsize))), key=lambda lp: getCostLoop(lp, fperm, fsize))
    unit = [d for d in range(len(p.size)) if p.size[d] == 1]
    return [[d for fd in lp for d in groups[fd]] + unit for lp in ranked[:limit]]


def grid_raster(desc: dict, order_fused: list) -> tuple:
    """The tile-grid raster (fused grid dimensions, fastest first) that an order of the fused
    dimensions gives a tile plan: the dimensions the tile covers whole do not step the grid."""
    fu, t = desc["fused"], desc.get("tile") or {}
    ext = t.get("ext") or [0] * fu["rank"]
    return tuple(d for d in order_fused if not (ext[d] and ext[d] == fu["size"][d]))


def preset_order(desc: dict, loop_order: int) -> list:
    """The fused-dimension order of a preset loop_order value (0 resolves to the planner's choice)."""
    fu = desc["fused"]
    lo = loop_order or desc.get("loop_order", 3)
    if lo == 1:
        return list(fu["perm"])
    if lo == 2:
        return list(range(fu["rank"]))[::-1]
    return list(range(fu["rank"]))


def plan_signature(desc: dict) -> tuple:
    t = desc.get("tile") or desc.get("row") or {}
    return (desc["kernel"], desc["vecA"], desc["vecB"], t.get("P", t.get("w")), t.get("LA"), t.get("LB"),
            t.get("ntiles", t.get("units")))


def tile_shapes(p: Problem, space: Optional[dict] = None) -> list[tuple[dict, dict]]:
    """Distinct plans the shape knobs (tile_elems x run_bytes) produce: [(shape knobs, shape-only
    plan json)], all planned in one host call without descriptor tables."""
    space = space or knob_space(p.dtype)
    tunings = [{k: v for k, v in (("tile_elems", te), ("run_bytes", rb)) if v}
               for te, rb in itertools.product(space["tile_elems"], space["run_bytes"])]
    descs = plan_shapes(p.perm, p.size, p.dtype, p.beta_nonzero, p.lda, p.ldb, tunings)
    seen = {}
    for tu, desc in zip(tunings, descs):
        if desc is None:
            continue
        sig = plan_signature(desc)
        if sig not in seen:
            seen[sig] = (tu, desc)
    return sorted(seen.values(), key=lambda x: (x[1]["est_cost"], len(x[0])))


def candidate_tunings(p: Problem, max_impl: int = 200, space: Optional[dict] = None,
                      with_desc: bool = False) -> list:
    """Distinct schedules for a problem, at most max_impl. The grid raster order, CTA count and tile
    kernel variant do not change the tile, so only the shape knobs are planned on the host.

    TTC keeps the best sqrt(maxImpl) blockings x sqrt(maxImpl) loop orders
    (GPUtransposeGenerator.py:220-230); here the tile shapes are ordered by the planner's estimate
    and taken round-robin, so every shape gets its default schedule before any gets a second one."""
    space = space or knob_space(p.dtype)
    rasters = space.get("rasters") or []
    explicit = []  # explicit loop orders (the caller's dimensions), TTC-ranked or given
    if isinstance(rasters, tuple) and rasters[0] == "ttc":
        explicit = ranked_loop_orders(p, max(rasters[1], int(math.ceil(math.sqrt(max(max_impl, 1))))))
        keep = rasters[1]
    else:
        explicit, keep = [list(r) for r in rasters], len(rasters)
    fused = fused_groups(p)[2] if explicit else None
    lists = []
    for shape_tu, desc in tile_shapes(p, space):
        if desc["kernel"] == "row":
            combos = [dict(shape_tu, blocks=b) if b else dict(shape_tu) for b in space["blocks"]]
        else:
            # the planner's raster choice (0) stands in for the explicit order it resolves to; an
            # explicit order joins only when its raster is one no earlier order gives
            orders, seen = [], set()
            for lo in space["loop_order"]:
                g = grid_raster(desc, preset_order(desc, lo))
                if g not in seen:
                    seen.add(g)
                    orders.append({"loop_order": lo} if lo else {})
            added = 0
            for order in explicit:
                if added >= keep:
                    break
                fo = []
                for d in order:
                    fd = next((i for i, grp in enumerate(fused) if d in grp), None)
                    if fd is not None and fd not in fo:
                        fo.append(fd)
                g = grid_raster(desc, fo)
                if g not in seen:
                    seen.add(g)
                    orders.append({"raster": list(order)})
                    added += 1
            combos = []
            for v, lo, b in itertools.product(space["tile_variant"], orders, space["blocks"]):
                tu = dict(shape_tu)
                tu.update(lo)
                for k, val in (("tile_variant", v), ("blocks", b)):
                    if val:
                        tu[k] = val
                combos.append(tu)
            # ring depth x CTAs per SM alternatives, on the first raster (the planner's, unless the
            # caller restricted the loop orders)
            for sch in schedule_alternatives(p, desc, space.get("schedules", 0)):
                combos.append(dict(shape_tu, **(orders[0] if orders else {}), **sch))
        lists.append([(tu, desc) for tu in combos])
    out = []
    depth = 0
    while len(out) < max(1, max_impl) and any(depth < len(l) for l in lists):
        for l in lists:
            if depth < len(l) and len(out) < max(1, max_impl):
                out.append(l[depth])
        depth += 1
    return out if with_desc else [tu for tu, _ in out]


class Bench:
    """Device buffers for timing one problem's candidates (allocated once per problem)."""

    def __init__(self, p: Problem, seed: int = 0):
        import torch
        self.p = p
        ta, tb = split_dtype(p.dtype)
        tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
        na, nb = p.buffer_elems()
        g = torch.Generator(device="cuda")
        g.manual_seed(seed)
        self.A = torch.rand(na, dtype=tmap[ta], device="cuda", generator=g)
        self.B0 = torch.rand(nb, dtype=tmap[tb], device="cuda", generator=g)
        self.B = self.B0.clone()
        self.ref = None
        self.flush_buf = L2Flush()

    def flush(self):
        self.flush_buf()

    def run_once(self, plan: Plan):
        self.B.copy_(self.B0)
        plan(self.A, self.B, self.p.alpha, self.p.beta)

    def time(self, plan: Plan, reps: int = 5, warmup: int = 1) -> float:
        import torch
        for _ in range(warmup):
            plan(self.A, self.B, self.p.alpha, self.p.beta)
        best = float("inf")
        small = self.p.bytes() < 2 * L2_BYTES
        for _ in range(reps):
            if small:
                self.flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            plan(self.A, self.B, self.p.alpha, self.p.beta)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best


def measure(p: Problem, tunings: Sequence[dict], reps: int = 5, verify: bool = True, seed: int = 0,
            bench: Optional[Bench] = None) -> list[Result]:
    """Times every tuning on one problem; with verify, checks each output against the first."""
    import torch
    bench = bench or Bench(p, seed)
    out = []
    for tu in tunings:
        plan = Plan(p.perm, p.size, p.dtype, p.beta_nonzero, p.lda, p.ldb, tu or None)
        ok = True
        if verify:
            bench.run_once(plan)
            if bench.ref is None:
                bench.ref = bench.B.clone()
            else:
                ok = bool(torch.equal(bench.B.view(torch.uint8), bench.ref.view(torch.uint8)))
        ms = bench.time(plan, reps)
        out.append(Result(dict(tu), ms, p.bytes() / (ms * 1e-3) / 1e9, plan.describe(), ok))
        plan.close()
    return out


def search(p: Problem, max_impl: int = 200, reps: int = 5, verify: bool = True, seed: int = 0) -> dict:
    """Exhaustive measured search. Returns {'best': Result, 'results': [...], 'seconds': wall}."""
    t0 = time.perf_counter()
    cands = candidate_tunings(p, max_impl)
    res = measure(p, cands, reps, verify, seed)
    bad = [r for r in res if not r.ok]
    if bad:
        raise RuntimeError(f"[TTC] ERROR: {len(bad)} schedules disagree with the first one: {bad[0].tuning}")
    best = min(res, key=lambda r: r.time_ms)
    return {"best": best, "results": res, "seconds": time.perf_counter() - t0, "candidates": len(cands)}


def batch_space(dtype: str) -> dict:
    """The knobs that matter inside the batched kernel: tile shape and raster order (it runs every
    complete tile through the staged asynchronous-copy layout on its own persistent grid, so the
    CTA count of a plain launch does not apply; candidates are timed with the staged kernel)."""
    base = 16384 // ELEM_BYTES[split_dtype(dtype)[0]]
    # tiles of at most half the default size: the batch's shared memory (and so its CTAs per SM) is
    # sized for its largest tile
    return {"tile_elems": [base // 4, base // 2], "run_bytes": [0, 256, 1024], "tile_variant": [3],
            "loop_order": [0, 1], "blocks": [0]}


def tune_for_batch(p: Problem, max_impl: int = 6, reps: int = 2, bench: Optional[Bench] = None) -> dict:
    """Measured search of one batched problem's schedule (timed with the table-driven kernel the
    batch runs). Returns the fastest tuning."""
    cands = candidate_tunings(p, max_impl, batch_space(p.dtype))
    if len(cands) <= 1:
        return cands[0] if cands else {}
    res = measure(p, cands, reps=reps, verify=False, bench=bench)
    return min(res, key=lambda r: r.time_ms).tuning
