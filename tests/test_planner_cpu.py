"""Host-side tests of the planner in libttcb200.so (no GPU): fast division, index fusion against
TTC's fuseIndices, validation errors, and a CPU replay of the kernels' index arithmetic from the
descriptor tables against the oracle's element mapping."""
import itertools
import json
import re
from pathlib import Path

import numpy as np
import pytest

import kernel_sim
import oracle.ttc_ref as ref
from ttc_b200 import TTCError, fuse, plan_host_json
from ttc_b200 import _native

ROOT = Path(__file__).resolve().parent.parent


def test_library_exports_every_header_symbol():
    declared = set()
    for header in sorted((ROOT / "include").glob("*.h")):
        declared |= set(re.findall(r"\b(ttcb_[a-z_]+)\s*\(", header.read_text()))
    declared -= {"ttcb_stream_t"}
    assert declared, "no declarations found"
    lib = _native.lib()
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    main = set(re.findall(r"\b(ttcb_[a-z_]+)\s*\(", (ROOT / "include" / "ttcb200.h").read_text()))
    assert main == {n for n, _, _ in _native.PUBLIC_SYMBOLS}


def test_fastdiv_matches_integer_division():
    rng = np.random.default_rng(0)
    divisors = list(range(1, 300)) + [int(x) for x in rng.integers(1, 2**31 - 1, 300)] + [2**k for k in range(31)]
    nums = [0, 1, 2, 3, 2**31 - 1, 2**31 - 2, 2**30] + [int(x) for x in rng.integers(0, 2**31 - 1, 40)]
    f = _native.lib().ttcb_test_fastdiv
    for d in divisors:
        for n in nums + [d - 1, d, d + 1, 3 * d, 3 * d - 1]:
            if 0 <= n < 2**31:
                assert f(n, d) == n // d, (n, d)
                assert int(kernel_sim.fdiv(n, (d, *_fd(d)))) == n // d


def _fd(d):
    l = 0
    while (1 << l) < d:
        l += 1
    m = ((((1 << l) - d) << 32) // d + 1) & 0xFFFFFFFF
    return m, l


def _random_problem(rng, max_rank=6, max_ext=9, pad=True, allow_one=False):
    r = int(rng.integers(1, max_rank + 1))
    lo = 1 if allow_one else 2
    size = [int(x) for x in rng.integers(lo, max_ext + 1, r)]
    perm = [int(x) for x in rng.permutation(r)]
    lda = ldb = None
    if pad and rng.random() < 0.5:
        lda = [s + int(rng.integers(0, 3)) for s in size]
    if pad and rng.random() < 0.5:
        ldb = [size[p] + int(rng.integers(0, 3)) for p in perm]
    return perm, size, lda, ldb


def test_fusion_matches_ttc_fuse_indices():
    rng = np.random.default_rng(1)
    for _ in range(400):
        perm, size, lda, ldb = _random_problem(rng, pad=True)
        sA, sB = ref.strides(size, perm, lda, ldb)
        fp, fn, fa, fb = fuse(perm, size, sA, sB)
        rs, rp, rla, rldb = ref.fuse_indices(size, perm, lda, ldb)
        rsA, rsB = ref.strides(rs, rp, rla, rldb)
        assert (fp, fn) == (rp, rs), (perm, size, lda, ldb)
        assert fa == rsA and fb == rsB, (perm, size, lda, ldb)


def _oracle_pairs(perm, size, lda, ldb):
    sA, sB = ref.strides(size, perm, lda, ldb)
    grids = np.meshgrid(*[np.arange(s, dtype=np.int64) for s in size], indexing="ij")
    a = sum(g * s for g, s in zip(grids, sA)).reshape(-1)
    b = sum(g * s for g, s in zip(grids, sB)).reshape(-1)
    return a, b


TUNINGS = [None, {"vec": 1}, {"loop_order": 1}, {"loop_order": 2}, {"tile_elems": 256}, {"tile_elems": 8192},
           {"run_bytes": 128}, {"run_bytes": 1024}, {"kernel": 1}, {"shifted_runs": 1}, {"bulk_copies": 1},
           {"bulk_copies": 1, "shifted_runs": 1}]


def test_kernel_index_math_replay_matches_oracle_mapping():
    rng = np.random.default_rng(2)
    n = 0
    for it in range(260):
        perm, size, lda, ldb = _random_problem(rng, max_rank=5, max_ext=13, allow_one=(it % 5 == 0))
        dtype = ["s", "d", "c", "z", "sd", "ds", "cz", "zc"][it % 8]
        tuning = TUNINGS[it % len(TUNINGS)]
        try:
            kind, (a, b) = kernel_sim.simulate(perm, size, dtype, bool(it % 2), lda, ldb, tuning)
        except TTCError:
            if tuning and tuning.get("kernel") == 1:
                continue  # some problems have no tile shape under a forced knob
            raise
        wa, wb = _oracle_pairs(perm, size, lda, ldb)
        assert len(b) == len(wb), (perm, size, lda, ldb, dtype, tuning)
        assert len(np.unique(b)) == len(b), "a B element is written twice"
        got = dict(zip(b.tolist(), a.tolist()))
        want = dict(zip(wb.tolist(), wa.tolist()))
        assert got == want, (perm, size, lda, ldb, dtype, tuning, kind)
        n += 1
    assert n > 200


@pytest.mark.parametrize("perm,size,lda,ldb", [
    ([1, 0, 2], [1000, 768, 16], None, None),
    ([3, 1, 0, 2], [96, 20, 18, 16], [104, 20, 19, 16], None),
    ([2, 0, 1], [7, 3, 3000], None, None),
    ([1, 0, 2], [20, 20, 700], None, None),
    ([0, 2, 1], [11, 8, 300], None, None),
    ([4, 2, 0, 3, 1], [9, 11, 7, 13, 5], None, None),
    ([0, 1, 2], [10, 20, 30], [12, 20, 30], [10, 22, 30]),
    # shared stride-1 rows of 512..1023 bytes go to the tile kernel
    ([0, 3, 2, 1], [156, 5, 7, 4], None, None),
    ([0, 2, 1], [130, 9, 11], [131, 9, 11], None),
])
def test_replay_larger_shapes(perm, size, lda, ldb):
    for tuning in (None, {"vec": 1}, {"loop_order": 1}):
        kind, (a, b) = kernel_sim.simulate(perm, size, "s", True, lda, ldb, tuning)
        wa, wb = _oracle_pairs(perm, size, lda, ldb)
        order = np.argsort(b)
        worder = np.argsort(wb)
        assert np.array_equal(b[order], wb[worder])
        assert np.array_equal(a[order], wa[worder])


def test_validation_errors():
    with pytest.raises(TTCError) as e:
        plan_host_json([0, 0, 1], [3, 4, 5])
    assert e.value.code == "TTCB_ERR_BAD_PERM"
    with pytest.raises(TTCError) as e:
        plan_host_json([1, 0], [3, 4], lda=[2, 4])
    assert e.value.code == "TTCB_ERR_BAD_LD"
    with pytest.raises(TTCError) as e:
        plan_host_json([1, 0], [3, 4], ldb=[3, 4])
    assert e.value.code == "TTCB_ERR_BAD_LD"
    with pytest.raises(TTCError) as e:
        plan_host_json(list(range(11)), [2] * 11)
    assert e.value.code == "TTCB_ERR_RANK"
    with pytest.raises(TTCError):
        plan_host_json([1, 0], [3, 4], dtype="sc")


def test_planner_choices_for_reference_shapes():
    j = plan_host_json([1, 0, 2], [1000, 768, 16], "s", True)
    assert j["kernel"] == "tile" and j["vecA"] == 4 and j["vecB"] == 4
    assert j["tile"]["LA"] * 4 >= 128 and j["tile"]["LB"] * 4 >= 128
    j = plan_host_json([0, 2, 1], [1000, 50, 60], "s", False)
    assert j["kernel"] == "row"
    j = plan_host_json([0, 1, 2], [10, 20, 30], "d", False)
    assert j["kernel"] == "row" and j["fused"]["rank"] == 1
    j = plan_host_json([1, 0, 2], [20, 20, 100000], "s", False)
    assert j["tile"]["LA"] >= 400 and j["tile"]["LB"] >= 400  # whole 20x20 planes per tile
    j = plan_host_json([3, 1, 0, 2], [96, 80, 72, 64], "zc", False, lda=[104, 80, 76, 64])
    assert j["kernel"] == "tile"
    # empty tensors are a no-op plan
    j = plan_host_json([1, 0], [0, 5], "s", False)
    assert j["elements"] == 0


def test_shape_only_plans_match_full_plans():
    """The learned selector plans its candidates shape-only and in one call (tile shapes enumerated
    once per problem); every candidate must describe the same tile, widths and cost as the full
    plan that the tuning produces."""
    import itertools
    from ttc_b200.core import plan_shapes
    rng = np.random.default_rng(7)
    tunings = [{k: v for k, v in (("tile_elems", te), ("run_bytes", rb), ("vec", vec)) if v}
               for te, rb, vec in itertools.product([0, 512, 2048, 8192], [0, 128, 1024], [0, 1])]
    for it in range(60):
        perm, size, lda, ldb = _random_problem(rng, max_rank=6, max_ext=40)
        dtype = ["s", "d", "zc", "sd"][it % 4]
        shapes = plan_shapes(perm, size, dtype, bool(it % 2), lda, ldb, tunings)
        for tu, sh in zip(tunings, shapes):
            try:
                full = plan_host_json(perm, size, dtype, bool(it % 2), lda, ldb, tu)
            except TTCError:
                assert sh is None
                continue
            assert sh is not None
            assert (sh["kernel"], sh["vecA"], sh["vecB"]) == (full["kernel"], full["vecA"], full["vecB"])
            assert abs(sh["est_cost"] - full["est_cost"]) <= 1e-9 * max(1.0, full["est_cost"])
            if full["kernel"] == "tile":
                for k in ("P", "LA", "LB", "ntiles", "ext"):
                    assert sh["tile"][k] == full["tile"][k], (perm, size, dtype, tu, k)


def test_ragged_tile_enumeration_covers_every_ragged_tile_once():
    """The staged kernel moves complete tiles only; the ragged-tile kernel enumerates the others by
    index (kernel_sim.simulate_tile checks the enumeration against a scan of every tile)."""
    rng = np.random.default_rng(2)
    primes = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53]  # no exact block sizes
    seen_two = seen_one = 0
    for it in range(300):
        r = int(rng.integers(2, 6))
        size = [int(rng.choice(primes)) for _ in range(r)]
        perm = [int(x) for x in rng.permutation(r)]
        for tu in (None, {"tile_elems": 256}, {"tile_elems": 64}):
            try:
                kind, b = kernel_sim.host_desc(perm, size, "s", False, None, None, tu)
            except TTCError:
                continue
            if kind != 1:
                continue
            t = kernel_sim.parse_tile(b)
            if t["nrag0"] > 0 and t["ntiles"] < 3000:
                kernel_sim.simulate_tile(t)
                seen_one += 1
                seen_two += t["nrag1"] > 0
    assert seen_one > 100 and seen_two > 5


def _pairs(a, b):
    return np.stack([np.asarray(a, np.int64), np.asarray(b, np.int64)], 1)


def test_edge_plans_move_exactly_the_ragged_tiles():
    """A plan's ragged tiles are moved as one or two boxes planned as transpositions of their own
    (edge plans, offset into A and B). Replaying each box's own plan must give exactly the element
    pairs (A read, B written) of the parent's ragged tiles, each once - with padded leading
    dimensions and a first fused stride other than 1 (a unit leading dimension in the box)."""
    rng = np.random.default_rng(11)
    primes = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53]
    checked = two = lead = 0
    for it in range(400):
        r = int(rng.integers(2, 6))
        size = [int(rng.choice(primes)) for _ in range(r)]
        perm = [int(x) for x in rng.permutation(r)]
        lda = ldb = None
        if it % 3 == 1:
            lda = [s + int(rng.integers(0, 3)) for s in size]
            ldb = [size[perm[j]] + int(rng.integers(0, 3)) for j in range(r)]
        if it % 5 == 2:
            # a unit first dimension with a padded leading dimension: fused stride 1 != 1
            size, perm = [1] + size, [0] + [x + 1 for x in perm]
            lda = [3] + (lda or size[1:])
            ldb = [1] + (ldb or [size[perm[j]] for j in range(1, r + 1)])
            r += 1
        dtype = ["s", "d", "zc"][it % 3]
        for tu in (None, {"tile_elems": 256}):
            try:
                kind, b = kernel_sim.host_desc(perm, size, dtype, False, lda, ldb, tu)
            except TTCError:
                continue
            if kind != 1:
                continue
            t = kernel_sim.parse_tile(b)
            if t["nrag0"] == 0 or t["ntiles"] > 3000:
                continue
            (af, bf), (ar, br) = kernel_sim.simulate_tile(t, split=True)
            boxes = kernel_sim.edge_boxes(perm, size, dtype, False, lda, ldb, tu)
            assert len(boxes) == 1 + (t["nrag1"] > 0), boxes
            ea, eb = [], []
            for bx in boxes:
                assert all(bx["lda"][i] >= bx["size"][i] for i in range(bx["rank"]))
                assert all(bx["ldb"][j] >= bx["size"][bx["perm"][j]] for j in range(bx["rank"]))
                k2, (a2, b2) = kernel_sim.simulate(bx["perm"], bx["size"], dtype, False, bx["lda"], bx["ldb"])
                ea.append(a2 + bx["offA"])
                eb.append(b2 + bx["offB"])
                lead += bx["rank"] > len([s for s in size if s > 1]) and bx["size"][0] == 1
            got = _pairs(np.concatenate(ea), np.concatenate(eb))
            want = _pairs(ar, br)
            assert len(np.unique(got[:, 1])) == len(got), "an edge plan writes a B element twice"
            got = got[np.lexsort(got.T[::-1])]
            want = want[np.lexsort(want.T[::-1])]
            assert np.array_equal(got, want), (perm, size, lda, ldb, dtype, tu, boxes)
            checked += 1
            two += len(boxes) == 2
    assert checked > 100 and two > 5 and lead > 0, (checked, two, lead)


def test_planner_raster_choice():
    """loop_order 0 leaves the tile grid's raster to the planner: B-major when B's runs are under
    256 bytes and B exceeds 64 MiB, else A-major (3); an explicit knob value is kept."""
    from ttc_b200.core import plan_host_json
    big_short_b = ([4, 2, 1, 3, 0], [39, 4, 7, 153, 314])  # fp32, B runs of 24 elements, 209 MB
    d = plan_host_json(*big_short_b, "s", False)
    assert d["tile"]["LB"] * 4 < 256 and d["elements"] * 4 >= 64 << 20
    assert d["loop_order"] == 1, d
    small = ([4, 2, 1, 3, 0], [39, 4, 7, 15, 314])
    assert plan_host_json(*small, "s", False)["loop_order"] == 3
    long_b = ([1, 0], [20, 1310720])  # fp64; B's stride-1 dimension is A's long one
    d = plan_host_json(*long_b, "d", False)
    assert d["tile"]["LB"] * 8 >= 256 and d["loop_order"] == 3, d
    for lo in (1, 2, 3):
        assert plan_host_json(*big_short_b, "s", False, tuning={"loop_order": lo})["loop_order"] == lo


def test_candidate_rasters_name_each_order_once():
    """The search's raster candidates are the planner's choice (0) plus the two orders it did not
    choose: for a large problem with short B runs (planner: B-major) the explicit A-major order (3)
    is searched and B-major (1) is not repeated; for a small one the reverse."""
    from ttc_b200.autotune import Problem, candidate_tunings
    big = Problem([4, 2, 1, 3, 0], [39, 4, 7, 153, 314], "s", 1.0, 0.0)
    small = Problem([4, 2, 1, 3, 0], [39, 4, 7, 15, 314], "s", 1.0, 0.0)
    for p, chosen, other in ((big, 1, 3), (small, 3, 1)):
        cands = candidate_tunings(p, max_impl=500, with_desc=True)
        orders = {tu.get("loop_order", 0) for tu, d in cands if d["kernel"] == "tile" and d["loop_order"] == chosen}
        assert chosen not in orders and other in orders and 0 in orders and 2 in orders, (orders, chosen)
        assert len({json.dumps(tu, sort_keys=True) for tu, _ in cands}) == len(cands)


def test_explicit_loop_orders_become_the_tile_grid_raster():
    """TTC's --loopPerm (GPUtransposeGenerator.py:203-230; blockIdx decoded fastest first,
    CUDAtranspose.py:737-779) as an explicit raster: for the README shape, whose tile leaves all three
    dimensions in the grid, every one of the six orders yields exactly that raster; fused groups take
    the place of their first member, dimensions the tile covers whole leave the grid, and orders that
    are not permutations are refused."""
    import itertools
    from ttc_b200 import TTCError
    from ttc_b200.core import plan_host_json
    for order in itertools.permutations(range(3)):
        d = plan_host_json([1, 0, 2], [1000, 768, 16], "s", True, tuning={"raster": list(order)})
        assert d["loop_order"] == 4 and d["raster"] == list(order), (order, d["raster"], d["tile"]["ext"])
    # an extent-1 dimension (here 1) is dropped by the fusion, but the order still lists it
    d = plan_host_json([2, 0, 3, 1], [64, 1, 48, 40], "s", False, tuning={"raster": [3, 1, 2, 0]})
    fused_of = {0: 0, 2: 1, 3: 2}
    want = [fused_of[x] for x in (3, 2, 0)]
    ext = d["tile"]["ext"]
    want = [w for w in want if not (ext[w] and ext[w] == d["fused"]["size"][w])]
    assert d["raster"] == want, (d["raster"], want, ext)
    for bad in ([0, 0, 1], [0, 1], [0, 1, 3]):
        with pytest.raises(TTCError):
            plan_host_json([1, 0, 2], [10, 20, 30], "s", False, tuning={"raster": bad})


def test_search_adds_ttc_ranked_loop_orders():
    """With TTC's ranking switched on, the search adds up to two explicit loop orders per tile shape,
    taken cheapest first by ttc_util.getCostLoop, and only those whose raster no preset order gives."""
    from ttc_b200.autotune import (Problem, candidate_tunings, grid_raster, knob_space, preset_order,
                                   ranked_loop_orders, fused_groups)
    from ttc_b200.ttc_util import getCostLoop
    p = Problem([4, 2, 1, 3, 0], [39, 4, 7, 153, 314], "s", 1.0, 0.0)
    fperm, fsize, groups = fused_groups(p)
    ranked = ranked_loop_orders(p, 10)
    costs = []
    for o in ranked:
        fo = []
        for dd in o:
            fd = next(i for i, g in enumerate(groups) if dd in g)
            if fd not in fo:
                fo.append(fd)
        costs.append(getCostLoop(fo, fperm, fsize))
    assert costs == sorted(costs)
    cands = candidate_tunings(p, 500, knob_space("s", ttc_orders=2), with_desc=True)
    by_shape = {}
    for tu, d in cands:
        if d["kernel"] != "tile" or {"stages", "round_robin", "shifted_runs", "bulk_copies"} & set(tu):  # schedule alternatives reuse the first raster
            continue
        key = json.dumps({k: v for k, v in tu.items() if k in ("tile_elems", "run_bytes")}, sort_keys=True)
        by_shape.setdefault(key, (d, []))[1].append(tu)
    assert any("raster" in tu for _, tus in by_shape.values() for tu in tus)
    for d, tus in by_shape.values():
        rasters = []
        for tu in tus:
            if "raster" in tu:
                fo = []
                for dd in tu["raster"]:
                    fd = next(i for i, g in enumerate(groups) if dd in g)
                    if fd not in fo:
                        fo.append(fd)
                rasters.append(grid_raster(d, fo))
            else:
                rasters.append(grid_raster(d, preset_order(d, tu.get("loop_order", 0))))
        assert len(set(rasters)) == len(set(json.dumps(tu, sort_keys=True) for tu in tus if not tu.get("blocks")))


def test_shifted_a_runs_replay():
    """Shifted A runs (tuning shifted_runs = 1): for random problems whose A runs 16-byte accesses
    cannot reach directly, the CPU replay of the load phase, for every tile shift, must put into each
    gathered slot exactly the A element the store phase expects (kernel_sim.check_shifted_layout),
    and the element mapping must equal the oracle's."""
    rng = np.random.default_rng(11)
    shifted = 0
    for it in range(90):
        perm, size, lda, ldb = _random_problem(rng, max_rank=4, max_ext=24)
        for dtype in ("s", "d", "c"):
            tu = {"shifted_runs": 1}
            try:
                kind, b = kernel_sim.host_desc(perm, size, dtype, False, lda, ldb, tu)
            except TTCError:
                continue
            if kind != 1:
                continue
            t = kernel_sim.parse_tile(b)
            if not t["shiftA"]:
                continue
            shifted += 1
            j = plan_host_json(perm, size, dtype, False, lda, ldb, tu)
            kernel_sim.check_staged_layout(t, j["vecA"])
            _, (a, b) = kernel_sim.simulate(perm, size, dtype, False, lda, ldb, tu)
            wa, wb = _oracle_pairs(perm, size, lda, ldb)
            assert dict(zip(b.tolist(), a.tolist())) == dict(zip(wb.tolist(), wa.tolist()))
    assert shifted >= 30


def test_bulk_copy_layout_replay():
    """Bulk A copies (asked for by bulk_copies = 1, alone and with shifted runs, and the planner's own
    choice): for random problems, the CPU replay of warp 0's bulk copies (kernel_sim.check_bulk_layout)
    must keep every copy on 16-byte boundaries and inside its stage, cut runs into pieces only at the
    padding points, and bring every element the store phase gathers; plans whose runs allow no bulk
    copy must not ask for them; and the element mapping must equal the oracle's."""
    rng = np.random.default_rng(12)
    seen = {0: 0, 1: 0}
    pieces = 0
    for it in range(70):
        # every other problem rank 2 with long extents (long runs, cut into pieces)
        perm, size, lda, ldb = _random_problem(rng, max_rank=4, max_ext=24) if it % 2 else \
            _random_problem(rng, max_rank=2, max_ext=600)
        for dtype in ("s", "d", "c", "z", "sd"):
            for tu in ({"bulk_copies": 1}, {"bulk_copies": 1, "shifted_runs": 1}, None):
                try:
                    kind, b = kernel_sim.host_desc(perm, size, dtype, False, lda, ldb, tu)
                except TTCError:
                    continue
                if kind != 1:
                    continue
                t = kernel_sim.parse_tile(b)
                j = plan_host_json(perm, size, dtype, False, lda, ldb, tu)
                EA = {"s": 4, "d": 8, "c": 8, "z": 16}[dtype[0]]
                if not t["bulkA"]:
                    assert tu is None or (not t["shiftA"] and j["vecA"] * EA != 16)
                    continue
                seen[t["shiftA"]] += 1
                pieces += int(t["bulk_pieces"] > 1)
                kernel_sim.check_bulk_layout(t, EA)
                kernel_sim.check_staged_layout(t, j["vecA"])
                _, (a, bb) = kernel_sim.simulate(perm, size, dtype, False, lda, ldb, tu)
                wa, wb = _oracle_pairs(perm, size, lda, ldb)
                assert dict(zip(bb.tolist(), a.tolist())) == dict(zip(wb.tolist(), wa.tolist()))
    assert seen[0] >= 40 and seen[1] >= 20 and pieces >= 5, (seen, pieces)


def test_lane_maps():
    """Lane maps of the staged kernel's register path (a warp takes B vectors from several B runs,
    in their natural order or sorted by A position, when that lowers the gather's bank conflicts):
    on random problems, every map is a bijection of the tile's B vectors whose lane groups each
    write whole 32-byte sectors of one B run, and every run order a permutation
    (kernel_sim.check_lane_map); without lane_map = 1 no plan has one; and the element mapping
    equals the oracle's."""
    rng = np.random.default_rng(21)
    maps = sorted_runs = 0
    for it in range(120):
        perm, size, lda, ldb = _random_problem(rng, max_rank=5, max_ext=40, pad=False)
        for dtype in ("s", "d", "sd"):
            try:
                kind, b = kernel_sim.host_desc(perm, size, dtype, it % 2 == 1, tuning={"lane_map": 1})
            except TTCError:
                continue
            if kind != 1:
                continue
            t = kernel_sim.parse_tile(b)
            if t["map_log2s"] < 0:
                continue
            maps += 1
            sorted_runs += int(t["runs"] is not None)
            EB = {"s": 4, "d": 8}[dtype[-1]]
            kernel_sim.check_lane_map(t, EB)
            _, b2 = kernel_sim.host_desc(perm, size, dtype, it % 2 == 1)
            assert kernel_sim.parse_tile(b2)["map_log2s"] < 0
            if maps <= 12:
                _, (a, bb) = kernel_sim.simulate(perm, size, dtype, it % 2 == 1, tuning={"lane_map": 1})
                wa, wb = _oracle_pairs(perm, size, None, None)
                assert dict(zip(bb.tolist(), a.tolist())) == dict(zip(wb.tolist(), wa.tolist()))
    assert maps >= 10 and sorted_runs >= 2, (maps, sorted_runs)
