"""CPU replay of the kernels' index arithmetic from a plan's descriptor bytes.

The planner (libttcb200.so, host code) emits the same descriptor the GPU kernels read. This module
parses it and replays, in numpy, which A element each kernel reads and which B element it writes -
tile decode, ragged limits, A/B run segments, shared-memory slots, row-copy units. Tests compare the
resulting element mapping with the oracle's, so the index math is checked without a GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ttc_b200 import _native
from ttc_b200._native import Tuning, i32, i64

_layout = None


def layout():
    global _layout
    if _layout is None:
        a = (ctypes.c_int64 * 13)()
        _native.lib().ttcb_test_desc_layout(a)
        keys = ["tile_size", "off_divLA", "off_g", "g_size", "off_bd", "bd_size", "row_size", "row_off_div",
                "row_off_sA", "row_off_sB", "fastdiv_size", "g_strideA", "off_shiftA"]
        _layout = dict(zip(keys, list(a)))
    return _layout


def host_desc(perm, size, dtype="s", beta=False, lda=None, ldb=None, tuning=None):
    """Returns (kernel kind, descriptor bytes) from the host-only planner."""
    ta, tb = (dtype[0], dtype[1]) if len(dtype) == 2 else (dtype, dtype)
    if isinstance(tuning, dict):
        tuning = Tuning.make(**tuning)
    kind = ctypes.c_int()
    args = (len(size), i32(perm), i64(size), i64(lda) if lda else None, i64(ldb) if ldb else None,
            _native.DTYPES[ta], _native.DTYPES[tb], int(beta), ctypes.byref(tuning) if tuning else None,
            ctypes.byref(kind))
    n = _native.lib().ttcb_test_plan_host_desc(*args, None, 0)
    if n == 0:
        raise _native.TTCError(1, _native.last_error())
    buf = ctypes.create_string_buffer(n)
    _native.lib().ttcb_test_plan_host_desc(*args, buf, n)
    return kind.value, buf.raw


def edge_boxes(perm, size, dtype="s", beta=False, lda=None, ldb=None, tuning=None):
    """The boxes a plan's ragged tiles are moved as (edge plans), from the host-only planner."""
    import json
    ta, tb = (dtype[0], dtype[1]) if len(dtype) == 2 else (dtype, dtype)
    if isinstance(tuning, dict):
        tuning = Tuning.make(**tuning)
    args = (len(size), i32(perm), i64(size), i64(lda) if lda else None, i64(ldb) if ldb else None,
            _native.DTYPES[ta], _native.DTYPES[tb], int(beta), ctypes.byref(tuning) if tuning else None)
    n = _native.lib().ttcb_test_plan_edges(*args, None, 0)
    if n == 0:
        raise _native.TTCError(1, _native.last_error())
    buf = ctypes.create_string_buffer(n)
    _native.lib().ttcb_test_plan_edges(*args, buf, n)
    return json.loads(buf.value.decode())


def _i32(b, off):
    return int(np.frombuffer(b, dtype=np.int32, count=1, offset=off)[0])


def _i64(b, off):
    return int(np.frombuffer(b, dtype=np.int64, count=1, offset=off)[0])


def _fd(b, off):
    d, m, l, _ = np.frombuffer(b, dtype=np.uint32, count=4, offset=off)
    return int(d), int(m), int(l)


def fdiv(n, fd):
    """The kernels' division by invariant integer, bit for bit (32-bit arithmetic)."""
    d, m, l = fd
    n = np.asarray(n, dtype=np.uint64)
    hi = (n * np.uint64(m)) >> np.uint64(32)
    return ((hi + n) & np.uint64(0xFFFFFFFF)) >> np.uint64(l)


def parse_tile(b):
    L = layout()
    names = ["P", "LA", "LB", "nsegA", "nsegB", "pshift", "pad", "phys_size", "ngrid", "nblocked", "ntiles",
             "off_segA", "off_segB", "off_perm", "smem_bytes", "fast", "async_ok", "padA", "stage_elems",
             "nstages", "off_gtab", "sigmaA", "reg_ok", "rag_a", "rag_b", "nrag0", "nrag1", "nfull"]
    t = {k: _i32(b, 4 * i) for i, k in enumerate(names)}
    t["divLA"] = _fd(b, L["off_divLA"])
    t["divLB"] = _fd(b, L["off_divLA"] + L["fastdiv_size"])
    g = []
    for k in range(t["ngrid"]):
        o = L["off_g"] + k * L["g_size"]
        g.append({"div": _fd(b, o), "divf": _fd(b, o + L["fastdiv_size"]), "strideA": _i64(b, o + L["g_strideA"]),
                  "strideB": _i64(b, o + L["g_strideA"] + 8), "n": _i64(b, o + L["g_strideA"] + 16),
                  "e": _i32(b, o + L["g_strideA"] + 24), "blocked": _i32(b, o + L["g_strideA"] + 28)})
    t["g"] = g
    bd = []
    for k in range(t["nblocked"]):
        o = L["off_bd"] + k * L["bd_size"]
        bd.append({"tsA": _fd(b, o), "tsB": _fd(b, o + 16), "ext": _fd(b, o + 32)})
    t["bd"] = bd
    t["segA"] = np.frombuffer(b, dtype=np.int64, count=t["nsegA"], offset=t["off_segA"])
    t["segB"] = np.frombuffer(b, dtype=np.int64, count=t["nsegB"], offset=t["off_segB"])
    t["ptab"] = np.frombuffer(b, dtype=np.uint16, count=t["P"], offset=t["off_perm"]).astype(np.int64)
    t["gtab"] = np.frombuffer(b, dtype=np.uint16, count=t["P"], offset=t["off_gtab"]).astype(np.int64)
    o = L["off_shiftA"]
    t["shiftA"], t["shiftW"], t["shiftCM"], t["bulkA"] = _i32(b, o), _i32(b, o + 4), _i32(b, o + 8), _i32(b, o + 12)
    t["bulk_pieces"] = _i32(b, o + 16 + L["fastdiv_size"])
    t["map_log2s"], t["map_nx"], t["map_nbx"] = (_i32(b, o + 20 + L["fastdiv_size"]), _i32(b, o + 24 + L["fastdiv_size"]),
                                                 _i32(b, o + 28 + L["fastdiv_size"]))
    t["divPieces"] = _fd(b, o + 32 + L["fastdiv_size"])
    t["map_vb"], t["map_ny"], t["map_nslots"] = (_i32(b, o + 32 + 2 * L["fastdiv_size"]),
                                                 _i32(b, o + 36 + 2 * L["fastdiv_size"]),
                                                 _i32(b, o + 40 + 2 * L["fastdiv_size"]))
    t["off_runs"] = _i32(b, o + 44 + 2 * L["fastdiv_size"])
    t["runs"] = (np.frombuffer(b, dtype=np.uint16, count=t["map_ny"], offset=t["off_runs"]).astype(np.int64)
                 if t["off_runs"] else None)
    return t


def lane_map_vectors(t, nslots):
    """The staged kernel's register-path lane map (TileDesc::map_log2s): the B vector that thread
    slot i (warp i / 32, lane i mod 32) takes, for i in 0..nslots-1 (-1: none)."""
    i = np.arange(nslots, dtype=np.int64)
    if t["map_log2s"] < 0:
        return np.where(i * max(t.get("map_vb", 1), 1) < t["P"], i, -1)
    ls, nbx, nx = t["map_log2s"], t["map_nbx"], t["map_nx"]
    w, l = i >> 5, i & 31
    y = (w // nbx) * (32 >> ls) + (l >> ls)
    ok = (y < t["map_ny"]) & (i < t["map_nslots"])
    run = y if t["runs"] is None else t["runs"][np.where(ok, y, 0)]
    v = (w % nbx) * (1 << ls) + (l & ((1 << ls) - 1)) + nx * run
    return np.where(ok, v, -1)


def check_lane_map(t, EB):
    """A lane map must give every B vector to exactly one thread slot within the register path's
    1024 slots, keep each group of map_s lanes on consecutive vectors of one B run, and give each
    group at least one whole 32-byte sector; the map's sizes must agree with the tile."""
    if t["map_log2s"] < 0:
        return
    vb = t["map_vb"]
    s = 1 << t["map_log2s"]
    nvB = t["P"] // vb
    rows = 32 // s
    assert t["LB"] % vb == 0 and t["map_nx"] == t["LB"] // vb and t["map_nbx"] * s == t["map_nx"]
    assert t["map_ny"] == t["P"] // t["LB"]
    assert t["map_nslots"] == t["map_nbx"] * ((t["map_ny"] + rows - 1) // rows) * 32 <= 1024
    assert s * vb * EB >= 32, "a lane group writes less than a 32-byte sector"
    if t["runs"] is not None:
        assert np.array_equal(np.sort(t["runs"]), np.arange(t["map_ny"])), "the run order is not a permutation"
    v = lane_map_vectors(t, 1024)
    got = v[v >= 0]
    assert np.array_equal(np.sort(got), np.arange(nvB)), "the lane map is not a bijection"
    g = v[: t["map_nslots"]].reshape(-1, s)
    g = g[g[:, 0] >= 0]
    assert (np.diff(g, axis=1) == 1).all() and ((g[:, 0] % t["map_nx"]) + s <= t["map_nx"]).all()


def check_bulk_layout(t, EA):
    """Bulk A copies (one cp.async.bulk per run, warp 0's lanes): replay the copies of a tile for
    every tile shift the kernel can meet and check that each starts and ends on 16-byte boundaries
    of shared memory and of A (tile bases included), stays inside its stage, and that the gather at
    gtab[q] (+ the shift) reads A element segA[s] + j of position p(q) = s*LA + j; and that the byte
    count announced to the stage barrier equals the bytes copied."""
    V = 16 // EA
    P, LA = t["P"], t["LA"]
    nseg = P // LA
    segA = t["segA"].astype(np.int64)
    q = np.arange(P, dtype=np.int64)
    slot_q = q + ((q >> t["pshift"]) if t["pad"] else 0)
    inv = np.full(t["phys_size"], -1, np.int64)
    inv[t["ptab"]] = np.arange(P, dtype=np.int64)
    p_of_q = inv[slot_q]
    want = segA[p_of_q // LA] + p_of_q % LA
    stage_bytes = ((t["stage_elems"] * EA + 15) // 16) * 16
    if not t["shiftA"]:
        m = t["bulk_pieces"]
        assert m >= 1 and LA % m == 0
        piece = LA // m
        if m == 1:
            assert t["sigmaA"] % LA == 0, "a padding point splits a run"
        else:
            assert t["sigmaA"] == piece, "pieces are not cut at the padding points"
        assert (piece * EA) % 16 == 0 and (segA * EA % 16 == 0).all()
        for g in t["g"]:
            assert (g["strideA"] * EA) % 16 == 0, "a tile base off the 16-byte grid"
        src = np.full(stage_bytes // EA + V, -(1 << 60), np.int64)
        total = 0
        for i in range(nseg * m):
            s = int(fdiv(i, t["divPieces"]))
            j = i - s * m
            assert s == i // m
            p = s * LA + j * piece
            dst = p + (p // t["sigmaA"]) * t["padA"]
            assert (dst * EA) % 16 == 0 and (dst + piece) * EA <= stage_bytes
            src[dst:dst + piece] = segA[s] + j * piece + np.arange(piece)
            total += piece * EA
        assert total == P * EA
        assert np.array_equal(src[t["gtab"]], want), "a gather reads an element no bulk copy brought"
        return
    W = t["shiftW"]
    assert W % V == 0
    for x in range(V):
        src = np.full(stage_bytes // EA + 2 * V, -(1 << 60), np.int64)
        total = 0
        for s in range(nseg):
            y = int(segA[s] % V)
            clo, chi = (x + y) // V, (x + y + LA - 1) // V
            dst = s * W + V * clo
            first = segA[s] - y + V * clo - x  # A element (from the tile base) of the copy's first slot
            n = (chi - clo + 1) * V
            assert ((first + x) * EA) % 16 == 0 and (dst * EA) % 16 == 0 and (dst + n) * EA <= stage_bytes
            # every 16-byte chunk of the copy holds an element of the run
            for c in range(clo, chi + 1):
                lo_el = segA[s] - y + V * c - x
                assert lo_el + V > segA[s] and lo_el < segA[s] + LA
            src[dst:dst + n] = first + np.arange(n)
            total += n * EA
        got = src[t["gtab"] + x]
        assert np.array_equal(got, want), f"shift {x}: a gather reads an element no bulk copy brought"


def check_shifted_layout(t, p_of_q, V):
    """Shifted A runs: for every tile shift x in 0..V-1, replay the load phase (chunk c of run s is
    copied when lo <= x < hi, from A element segA[s] - y + V*c - x past the tile base into slot
    s*W + V*c, y = segA[s] mod V) and check that the gather at gtab[q] + x finds A element
    segA[s] + j of position p(q) = s*LA + j, that every copied chunk overlaps its run (so no copy
    leaves the 16-byte blocks the run touches) and that nothing lies beyond the stage."""
    P, LA, W, CM = t["P"], t["LA"], t["shiftW"], t["shiftCM"]
    nseg = P // LA
    segA = t["segA"].astype(np.int64)
    y = segA % V
    assert W % V == 0 and W >= CM * V and nseg * W <= t["stage_elems"]
    for x in range(V):
        src = np.full(t["stage_elems"] + V, -(1 << 60), np.int64)
        for s in range(nseg):
            for c in range(CM):
                lo, hi = c * V - y[s] - LA + 1, (c + 1) * V - y[s]
                if not (lo <= x < hi):
                    continue
                first = segA[s] - y[s] + V * c - x  # A element (from the tile base) of the chunk's first slot
                assert first + V > segA[s] and first < segA[s] + LA, "a copied chunk misses its run"
                src[s * W + V * c: s * W + V * c + V] = first + np.arange(V)
        s_of, j_of = p_of_q // LA, p_of_q % LA
        got = src[t["gtab"] + x]
        assert np.array_equal(got, segA[s_of] + j_of), f"shift {x}: a gather reads an element it was not given"


def check_staged_layout(t, vecA):
    """The staged kernel's gather table must read, for B position q, the element that the load
    phase copied from A position p(q) (staged at p + (p // LA) * padA), with vector-aligned copies."""
    P = t["P"]
    q = np.arange(P, dtype=np.int64)
    slot_q = q + ((q >> t["pshift"]) if t["pad"] else 0)
    inv = np.full(t["phys_size"], -1, np.int64)
    inv[t["ptab"]] = np.arange(P, dtype=np.int64)
    p_of_q = inv[slot_q]
    assert (p_of_q >= 0).all()
    if t["shiftA"]:
        check_shifted_layout(t, p_of_q, vecA)
        return
    stg = p_of_q + (p_of_q // t["sigmaA"]) * t["padA"]
    assert np.array_equal(stg, t["gtab"]), "gtab disagrees with the staged layout"
    assert len(np.unique(t["gtab"])) == P and t["gtab"].max() < t["stage_elems"]
    assert t["stage_elems"] >= t["phys_size"]
    p = np.arange(0, P, vecA, dtype=np.int64)
    assert ((p + (p // t["sigmaA"]) * t["padA"]) % vecA == 0).all(), "staged vectors misaligned"
    # a vector never straddles a padding point
    assert t["sigmaA"] % vecA == 0


def parse_row(b):
    L = layout()
    r = {"w": _i64(b, 0), "chunk": _i32(b, 8), "nchunk": _i32(b, 12), "nd": _i32(b, 16), "nunits": _i32(b, 20),
         "divChunk": _fd(b, 24)}
    r["div"] = [_fd(b, L["row_off_div"] + 16 * k) for k in range(r["nd"])]
    r["sA"] = [_i64(b, L["row_off_sA"] + 8 * k) for k in range(r["nd"])]
    r["sB"] = [_i64(b, L["row_off_sB"] + 8 * k) for k in range(r["nd"])]
    return r


def simulate_tile(t, split=False):
    """Returns arrays (a_off, b_off): for every element written, the A element read. With split,
    returns them for the complete tiles and for the ragged tiles separately."""
    P = t["P"]
    p = np.arange(P, dtype=np.int64)
    q = np.arange(P, dtype=np.int64)
    slot_q = q + ((q >> t["pshift"]) if t["pad"] else 0)
    sA = fdiv(p, t["divLA"]).astype(np.int64)
    a_rel = t["segA"][sA] + (p - sA * t["LA"])
    sB = fdiv(q, t["divLB"]).astype(np.int64)
    b_rel = t["segB"][sB] + (q - sB * t["LB"])
    phys = int(slot_q.max()) + 1 if P else 0
    assert phys == t["phys_size"], (phys, t["phys_size"])
    assert len(np.unique(t["ptab"])) == P, "two elements share a shared-memory slot"
    assert set(t["ptab"].tolist()) == set(slot_q.tolist()), "load and store slots differ"
    a_out, b_out = [], []
    ragged = []
    is_rag = []
    for tile in range(t["ntiles"]):
        rem = tile
        bA = bB = 0
        lim = [1 << 31, 1 << 31]
        for g in t["g"]:
            qq = int(fdiv(rem, g["div"]))
            blk = rem - qq * g["div"][0]
            rem = qq
            bA += blk * g["strideA"]
            bB += blk * g["strideB"]
            if g["blocked"] >= 0:
                lim[g["blocked"]] = min(g["e"], g["n"] - blk * g["e"])
                if lim[g["blocked"]] < g["e"]:
                    ragged.append(tile)
        okA = np.ones(P, bool)
        okB = np.ones(P, bool)
        for k, bd in enumerate(t["bd"]):
            c = fdiv(p, bd["tsA"]).astype(np.int64)
            c = c - fdiv(c, bd["ext"]).astype(np.int64) * bd["ext"][0]
            okA &= c < lim[k]
            c = fdiv(q, bd["tsB"]).astype(np.int64)
            c = c - fdiv(c, bd["ext"]).astype(np.int64) * bd["ext"][0]
            okB &= c < lim[k]
        # slot -> A offset written in the load phase
        slot_to_a = np.full(phys, -1, np.int64)
        slot_to_a[t["ptab"][okA]] = bA + a_rel[okA]
        src = slot_to_a[slot_q[okB]]
        assert (src >= 0).all(), "store phase reads a slot the load phase did not write"
        a_out.append(src)
        b_out.append(bB + b_rel[okB])
        is_rag.append(bool(ragged) and ragged[-1] == tile)
    # the staged kernel walks the complete tiles, numbered over the divf counts
    full = []
    for tf in range(t["nfull"]):
        rem, tile, M = tf, 0, 1
        for g in t["g"]:
            qq = int(fdiv(rem, g["divf"]))
            tile += (rem - qq * g["divf"][0]) * M
            rem = qq
            M *= g["div"][0]
        full.append(tile)
    assert sorted(full) == sorted(set(range(t["ntiles"])) - set(ragged)), "complete-tile enumeration differs"
    # the ragged tiles go to the ragged-tile kernel, which enumerates them by index
    want = sorted(set(ragged))
    got = [ragged_tile_index(t, r) for r in range(t["nrag0"] + t["nrag1"])]
    assert len(got) == len(set(got)), "a ragged tile is enumerated twice"
    assert sorted(got) == want, "ragged-tile enumeration differs from the ragged tiles"
    if split:
        def cat(xs, keep):
            xs = [x for x, k in zip(xs, is_rag) if k == keep]
            return np.concatenate(xs) if xs else np.zeros(0, np.int64)
        return (cat(a_out, False), cat(b_out, False)), (cat(a_out, True), cat(b_out, True))
    return np.concatenate(a_out) if a_out else np.zeros(0, np.int64), \
        np.concatenate(b_out) if b_out else np.zeros(0, np.int64)


def ragged_tile_index(t, r):
    """The ragged-tile kernel's r -> tile index (mixed radix with the ragged dimension pinned)."""
    fixed, excl = t["rag_a"], -1
    if r >= t["nrag0"]:
        r -= t["nrag0"]
        fixed, excl = t["rag_b"], t["rag_a"]
    tile, M = 0, 1
    for k, g in enumerate(t["g"]):
        cnt = g["div"][0]
        if k == fixed:
            c = cnt - 1
        else:
            radix = cnt - 1 if k == excl else cnt
            c = r % radix
            r //= radix
        tile += c * M
        M *= cnt
    return tile


def simulate_row(r):
    a_out, b_out = [], []
    for u in range(r["nunits"]):
        row = int(fdiv(u, r["divChunk"]))
        ck = u - row * r["nchunk"]
        rem = row
        oA = oB = 0
        for k in range(r["nd"]):
            qq = int(fdiv(rem, r["div"][k]))
            c = rem - qq * r["div"][k][0]
            rem = qq
            oA += c * r["sA"][k]
            oB += c * r["sB"][k]
        e0 = ck * r["chunk"]
        e1 = min(e0 + r["chunk"], r["w"])
        e = np.arange(e0, e1, dtype=np.int64)
        a_out.append(oA + e)
        b_out.append(oB + e)
    return np.concatenate(a_out), np.concatenate(b_out)


def simulate(perm, size, dtype="s", beta=False, lda=None, ldb=None, tuning=None):
    kind, b = host_desc(perm, size, dtype, beta, lda, ldb, tuning)
    if kind == 1:
        t = parse_tile(b)
        if t["async_ok"]:
            import json
            from ttc_b200 import plan_host_json
            j = plan_host_json(perm, size, dtype, beta, lda, ldb, tuning)
            check_staged_layout(t, j["vecA"])
        return kind, simulate_tile(t)
    if kind == 2:
        return kind, simulate_row(parse_row(b))
    return kind, (np.zeros(0, np.int64), np.zeros(0, np.int64))
