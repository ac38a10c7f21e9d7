"""GPU parity: the sm_100a kernels against the CPU oracle, bit for bit.

Every kernel rounds each product and sum once (explicitly rounded intrinsics), like the oracle
compiled without contraction, so the bar is bit-exact for every dtype pair and alpha/beta - stricter
than the <= 1 ulp the contracted reference would allow.
"""
import numpy as np
import pytest

import oracle
from helpers import (assert_bitexact, make_inputs, split, ttc_cases, uniform, NP, buffer_len)

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def run_gpu(A, B, perm, size, dtype, alpha, beta, lda=None, ldb=None, tuning=None, offset=0):
    """Runs the library on copies of A and B; offset shifts both buffers by elements (alignment)."""
    torch = _torch()
    from ttc_b200 import Plan
    ta, tb = split(dtype)
    tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
    dA = torch.empty(A.size + offset, dtype=tmap[ta], device="cuda")
    dB = torch.empty(B.size + offset + 64, dtype=tmap[tb], device="cuda")
    dA[offset:].copy_(torch.from_numpy(A))
    dB[offset:offset + B.size].copy_(torch.from_numpy(B))
    canary = torch.from_numpy(uniform(64, tb, 99))
    dB[offset + B.size:].copy_(canary)
    plan = Plan(perm, size, dtype, complex(beta) != 0, lda, ldb, tuning)
    plan(dA[offset:], dB[offset:], alpha, beta)
    torch.cuda.synchronize()
    out = dB[offset:offset + B.size].cpu().numpy()
    tail = dB[offset + B.size:].cpu().numpy()
    assert np.array_equal(tail.view(np.uint8), canary.numpy().view(np.uint8)), "write past the end of B"
    desc = plan.describe()
    assert plan.wait_timeouts() == 0, "a stage wait of the bulk-copy kernel ran out of time"
    plan.close()
    return out, desc


def check_case(perm, size, dtype, alpha, beta, lda=None, ldb=None, tuning=None, seed=7, offset=0):
    A, B = make_inputs(size, perm, dtype, seed, lda, ldb)
    want = oracle.transpose(A, B.copy(), perm, size, alpha, beta, lda, ldb, dtype)
    got, desc = run_gpu(A, B, perm, size, dtype, alpha, beta, lda, ldb, tuning, offset)
    assert_bitexact(got, want, f"perm={perm} size={size} dtype={dtype} a={alpha} b={beta} lda={lda} "
                               f"ldb={ldb} tuning={tuning} plan={desc}")
    return desc


def test_ttc_reference_case_matrix():
    """The reference's own sweep (test-framework/ttc_test.py:80-217) on the GPU path."""
    for perm, size, dtype, alpha, beta in ttc_cases():
        check_case(perm, size, dtype, alpha, beta)


def test_against_ttc_golden_fixtures():
    """The GPU path against the outputs of TTC's own generated reference loop (tests/golden)."""
    import json
    from pathlib import Path
    z = np.load(Path(__file__).resolve().parent / "golden" / "ttc_reference_loop.npz")
    cases = json.loads(bytes(z["meta"]).decode())["cases"]
    for k, c in enumerate(cases):
        A, B = make_inputs(c["size"], c["perm"], c["dtype"], c["seed"], c["lda"], c["ldb"])
        for tuning in (None, {"tile_variant": 1}, {"tile_variant": 2}):
            got, desc = run_gpu(A, B, c["perm"], c["size"], c["dtype"], c["alpha"], c["beta"], c["lda"], c["ldb"],
                                tuning)
            assert_bitexact(got, z[f"B{k}"], f"golden {k} {c} tuning={tuning} plan={desc}")


def test_readme_shape_full_size():
    """perm 1,0,2 / 1000x768x16 fp32, alpha = beta = 1 (the README example)."""
    desc = check_case([1, 0, 2], [1000, 768, 16], "s", 1.0, 1.0)
    assert desc["kernel"] == "tile"
    check_case([1, 0, 2], [1000, 768, 16], "s", 1.0, 0.0)


@pytest.mark.parametrize("dtype,alpha", [("zc", complex(0.5, 0.25)), ("ds", 0.5), ("z", complex(0.5, 0.25)),
                                         ("d", 0.5)])
def test_strided_mixed_precision_config(dtype, alpha):
    """rank-4 perm 3,1,0,2, extents 96,80,72,64, lda = extents + {8,0,4,0}, B dense, beta = 0."""
    check_case([3, 1, 0, 2], [96, 80, 72, 64], dtype, alpha, 0.0, lda=[104, 80, 76, 64])


@pytest.mark.parametrize("dtype", ["s", "d", "c", "z", "sd", "ds", "cz", "zc"])
def test_padded_lda_ldb_and_complex_beta(dtype):
    ta, tb = split(dtype)
    cplx = ta in "cz"
    alpha = complex(1.25, -0.75) if cplx else 1.25
    beta = complex(-0.5, 0.3) if cplx else -0.5
    check_case([2, 0, 3, 1], [13, 9, 6, 11], dtype, alpha, beta, lda=[16, 10, 6, 12], ldb=[6, 15, 12, 9])
    check_case([1, 2, 0], [33, 17, 9], dtype, alpha, 0.0, ldb=[17, 12, 33])


TUNINGS = [{"vec": 1}, {"loop_order": 1}, {"loop_order": 2}, {"loop_order": 3}, {"blocks": 7}, {"tile_elems": 512},
           {"tile_elems": 8192}, {"run_bytes": 128}, {"run_bytes": 2048}, {"kernel": 1}, {"streaming": -1},
           {"streaming": 1}, {"round_robin": 1}, {"stages": 3}, {"stages": 7}, {"ctas_per_sm": 1},
           {"stages": 6, "ctas_per_sm": 2}, {"round_robin": 1, "blocks": 5}, {"round_robin": -1},
           {"round_robin": -1, "blocks": 5}, {"round_robin": -1, "claim_group": 3},
           {"round_robin": -1, "claim_group": 8, "blocks": 3}, {"bulk_copies": 1}, {"bulk_copies": 1, "round_robin": -1},
           {"bulk_copies": 1, "shifted_runs": 1}, {"lane_map": 1}]


@pytest.mark.parametrize("tuning", TUNINGS, ids=[str(t) for t in TUNINGS])
def test_schedule_knobs_do_not_change_results(tuning):
    for perm, size in ([[1, 0, 2], [300, 257, 5]], [[2, 0, 1], [7, 3, 20001]], [[0, 2, 1], [40, 33, 17]],
                       [[4, 2, 0, 3, 1], [9, 11, 7, 13, 5]], [[0, 1], [1000, 77]]):
        for dtype, beta in (("s", 0.0), ("d", 1.5), ("c", 0.0)):
            try:
                check_case(perm, size, dtype, 1.5, beta, tuning=tuning)
            except Exception as e:  # a forced tile kernel may not apply to every problem
                if "TTCB_ERR_UNSUPPORTED" in str(e) and tuning.get("kernel"):
                    continue
                raise


@pytest.mark.parametrize("order", [[0, 1, 2], [0, 2, 1], [1, 0, 2], [1, 2, 0], [2, 0, 1], [2, 1, 0]])
def test_every_explicit_loop_order(order):
    """TTC's --loopPerm as the tile grid's raster: each of the six orders of a rank-3 problem whose
    tile leaves every dimension in the grid, with ragged blocks, for beta = 0 and beta != 0."""
    for dtype, beta in (("s", 0.0), ("d", -0.5)):
        desc = check_case([1, 0, 2], [301, 263, 7], dtype, 1.5, beta, tuning={"raster": order})
        assert desc["loop_order"] == 4


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_misaligned_pointers_fall_back_to_narrow_accesses(offset):
    check_case([1, 0, 2], [64, 96, 3], "s", 1.0, 0.5, offset=offset)
    check_case([0, 2, 1], [256, 7, 9], "s", 2.0, 0.0, offset=offset)
    check_case([1, 0], [40, 33], "d", 1.0, 1.0, offset=offset)


def test_random_problems_ranks_1_to_6():
    rng = np.random.default_rng(11)
    for it in range(120):
        r = int(rng.integers(1, 7))
        size = [int(x) for x in rng.integers(1, 14, r)]
        perm = [int(x) for x in rng.permutation(r)]
        dtype = ["s", "d", "c", "z", "sd", "ds", "cz", "zc"][it % 8]
        beta = [0.0, 1.0, -0.5][it % 3]
        lda = [s + int(rng.integers(0, 2)) for s in size] if it % 4 == 0 else None
        check_case(perm, size, dtype, 1.5, beta, lda=lda, seed=it)


def test_edge_values_and_signed_zero():
    """Values that expose sign, rounding and special-value handling (NaN, inf, -0, denormals)."""
    torch = _torch()
    perm, size = [1, 0], [37, 41]
    for dtype in ("s", "d", "ds", "sd"):
        ta, tb = split(dtype)
        A, B = make_inputs(size, perm, dtype, 3)
        special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-40, -1e-310, 3.4e38, 1.0 + 2**-23],
                           dtype=np.float64)
        A[: special.size] = special.astype(A.dtype)
        B[-special.size:] = special.astype(B.dtype)
        for alpha, beta in ((1.0, 0.0), (-1.0, 1.0), (3.0, -2.0)):
            want = oracle.transpose(A, B.copy(), perm, size, alpha, beta, dtype=dtype)
            got, _ = run_gpu(A, B, perm, size, dtype, alpha, beta)
            assert_bitexact(got, want, f"special {dtype} {alpha} {beta}")


def test_empty_and_single_element():
    check_case([0], [1], "s", 2.0, 1.0)
    check_case([1, 0], [1, 1], "z", complex(2, 1), 0.0)
    from ttc_b200 import Plan
    torch = _torch()
    p = Plan([1, 0], [0, 5], "s")
    x = torch.zeros(4, device="cuda")
    p(x, x, 1.0)  # no-op
    torch.cuda.synchronize()


def test_error_paths_do_not_poison_the_context():
    import ctypes
    from ttc_b200 import Plan, TTCError
    from ttc_b200._native import check, lib
    torch = _torch()
    x = torch.zeros(64, device="cuda")
    y = torch.zeros(64, device="cuda")
    p0 = Plan([1, 0], [8, 8], "s", beta_nonzero=False)
    with pytest.raises(TTCError) as e:
        p0(x, y, 1.0, 0.5)  # beta given to a plan made for beta == 0
    assert e.value.code == "TTCB_ERR_BETA"
    with pytest.raises(TTCError) as e:
        Plan([1, 0], [8, 8], "s", lda=[4, 8])
    assert e.value.code == "TTCB_ERR_BAD_LD"
    with pytest.raises(TTCError) as e:
        Plan([0, 0], [8, 8], "s")
    assert e.value.code == "TTCB_ERR_BAD_PERM"
    al = (ctypes.c_float * 1)(1.0)
    with pytest.raises(TTCError) as e:  # A not aligned to its element size
        check(lib().ttcb_transpose(p0.handle, x.data_ptr() + 2, y.data_ptr(), ctypes.cast(al, ctypes.c_void_p),
                                   None, None))
    assert e.value.code == "TTCB_ERR_ALIGN"
    p1 = Plan([1, 0], [8, 8], "s", beta_nonzero=True)
    with pytest.raises(TTCError) as e:  # beta missing for a beta != 0 plan
        check(lib().ttcb_transpose(p1.handle, x.data_ptr(), y.data_ptr(), ctypes.cast(al, ctypes.c_void_p),
                                   None, None))
    assert e.value.code == "TTCB_ERR_BETA"
    # the context is still healthy
    check_case([1, 0], [8, 8], "s", 1.0, 0.0)


def test_torch_permute_agrees_on_large_sweep_shapes():
    """Size-independent property at full size: for alpha = 1, beta = 0 the result is a pure
    permutation, identical to torch.permute(...).contiguous() bit for bit."""
    torch = _torch()
    from ttc_b200 import Plan
    import ttc_b200.workloads as wl
    cases = wl.sweep_cases(seed=2024)[:6]
    rasters, edges = set(), 0
    for c in cases:
        size, perm = c["size"], c["perm"]
        tdt = torch.float32 if c["dtype"] == "s" else torch.float64
        n = int(np.prod(size))
        A = torch.rand(n, dtype=tdt, device="cuda") * 2 - 1
        B = torch.empty_like(A)
        p = Plan(perm, size, c["dtype"], False)
        p(A, B, 1.0, 0.0)
        # A viewed row-major with reversed dims; B's dims are A's dims in perm order
        At = A.view(*reversed(size))
        nd = len(size)
        want = At.permute(*[nd - 1 - perm[j] for j in reversed(range(nd))]).contiguous().view(-1)
        torch.cuda.synchronize()
        assert torch.equal(B, want), (perm, size, p.describe())
        d = p.describe()
        rasters.add(d["loop_order"])
        edges += bool(d.get("edges"))
        del A, B, At, want
        torch.cuda.empty_cache()
    # the planner's raster choice (B-major for short B runs) and edge plans are both exercised
    assert rasters == {1, 3} and edges > 0, (rasters, edges)


@pytest.mark.parametrize("perm,size", [([1, 0], [46341, 46341]), ([2, 0, 1], [3, 65537, 10923])])
def test_more_than_2_to_the_31_elements(perm, size):
    """Maximum sizes: tensors with more than 2^31 elements (8.6 GB each in fp32) need 64-bit tile
    bases (TTC used int everywhere). alpha = 1, beta = 0 is a pure permutation, compared with
    torch.permute(...).contiguous() bit for bit on the GPU."""
    torch = _torch()
    from ttc_b200 import Plan
    n = int(np.prod(size))
    assert n > 2**31
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    A = torch.rand(n, device="cuda", generator=g)
    B = torch.empty_like(A)
    p = Plan(perm, size, "s", False)
    p(A, B, 1.0, 0.0)
    nd = len(size)
    want = A.view(*reversed(size)).permute(*[nd - 1 - perm[j] for j in reversed(range(nd))]).contiguous().view(-1)
    torch.cuda.synchronize()
    assert torch.equal(B, want), (perm, size, p.describe())
    p.close()
    del A, B, want
    torch.cuda.empty_cache()


@pytest.mark.parametrize("ragged", [0, 1])
@pytest.mark.parametrize("dtype,beta", [("s", 0.0), ("d", -0.5), ("zc", 0.0)])
def test_ragged_tiles_beside_the_staged_kernel_streams_and_graphs(dtype, beta, ragged):
    """Prime extents leave ragged last blocks: the staged kernel moves the complete tiles while the
    side stream, forked from the caller's stream and joined back, moves the rest - as edge plans
    (the ragged boxes planned as transpositions of their own, offset into A and B) or, with the
    `ragged` knob at 1, with the element-wise ragged-tile kernel. The result must equal the oracle
    when called on the default stream, on a side torch stream, and when the call is captured into
    a CUDA graph and replayed (the fork and join are captured with it)."""
    torch = _torch()
    from ttc_b200 import Plan
    perm, size = [2, 0, 1], [67, 131, 251]
    ta, tb = split(dtype)
    tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
    A, B = make_inputs(size, perm, dtype, 31)
    want = oracle.transpose(A, B.copy(), perm, size, 1.5, beta, dtype=dtype)
    plan = Plan(perm, size, dtype, beta != 0, tuning={"ragged": ragged})
    d = plan.describe()
    t = d["tile"]
    assert t["async"] == 1 and t["ragged_tiles"] > 0, t
    assert bool(d.get("edges")) == (ragged == 0), d
    dA = torch.from_numpy(A).cuda()
    for mode in ("default", "stream", "graph"):
        dB = torch.from_numpy(B.copy()).cuda()
        if mode == "default":
            plan(dA, dB, 1.5, beta)
        elif mode == "stream":
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                plan(dA, dB, 1.5, beta, s)
            torch.cuda.current_stream().wait_stream(s)
        else:
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    plan(dA, dB, 1.5, beta, s)
            dB.copy_(torch.from_numpy(B))
            g.replay()
        torch.cuda.synchronize()
        assert_bitexact(dB.cpu().numpy(), want, f"{mode} {dtype} beta={beta} tile={t}")
    plan.close()


@pytest.mark.parametrize("offset", [0, 1])
def test_edge_plans_random_ragged_problems(offset):
    """Problems whose tiles leave ragged last blocks (prime extents), with padded lda/ldb, a unit
    first dimension with a padded leading dimension (the edge boxes then start with a unit
    dimension), mixed and complex types, beta != 0 and misaligned base pointers: the edge plans
    (offset sub-problems moved by the staged kernel on the side stream) must give the oracle's
    result bit for bit."""
    rng = np.random.default_rng(23 + offset)
    primes = [3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67]
    with_edges = 0
    for it in range(48):
        r = int(rng.integers(2, 6))
        size = [int(rng.choice(primes)) for _ in range(r)]
        perm = [int(x) for x in rng.permutation(r)]
        while perm == sorted(perm):
            perm = [int(x) for x in rng.permutation(r)]
        lda = ldb = None
        if it % 3 == 1:
            lda = [s + int(rng.integers(0, 3)) for s in size]
            ldb = [size[perm[j]] + int(rng.integers(0, 3)) for j in range(r)]
        if it % 4 == 2:
            size, perm = [1] + size, [0] + [x + 1 for x in perm]
            lda = [2] + (lda or size[1:])
            ldb = [1] + (ldb or [size[perm[j]] for j in range(1, r + 1)])
        dtype = ["s", "d", "zc", "ds", "c"][it % 5]
        beta = [0.0, -0.5][it % 2]
        tuning = {"tile_elems": [0, 256, 512][it % 3]} if it % 3 else None
        desc = check_case(perm, size, dtype, 1.5, beta, lda, ldb, tuning, seed=100 + it, offset=offset)
        with_edges += bool(desc.get("edges"))
    assert with_edges >= 12, with_edges


def test_claimed_tiles_with_concurrent_launches_and_slot_reuse():
    """The staged kernel's tiles claimed from the plan's counters: one plan launched on four streams
    at once (different counter slots), then 150 launches in a row on one stream (every slot used and
    reset more than twice), each result bit for bit equal to the oracle's."""
    import torch
    from ttc_b200 import Plan
    perm, size = [2, 0, 1], [67, 45, 311]
    plan = Plan(perm, size, "s", True, tuning={"blocks": 16, "round_robin": -1})
    assert plan.describe()["tile"]["async"] == 1 and plan.describe()["tile"]["claims"] == 1
    n = int(np.prod(size))
    streams = [torch.cuda.Stream() for _ in range(4)]
    ins, outs, wants = [], [], []
    for k in range(4):
        A, B = make_inputs(size, perm, "s", 300 + k)
        wants.append(oracle.transpose(A, B.copy(), perm, size, 1.5, -0.5, dtype="s"))
        ins.append(torch.from_numpy(A).cuda())
        outs.append(torch.from_numpy(B).cuda())
    torch.cuda.synchronize()
    for k, st in enumerate(streams):
        plan(ins[k], outs[k], 1.5, -0.5, st)
    torch.cuda.synchronize()
    for k in range(4):
        assert_bitexact(outs[k].cpu().numpy(), wants[k], f"stream {k}")
    A, B = make_inputs(size, perm, "s", 400)
    want = B.copy()
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    for rep in range(150):
        plan(dA, dB, 1.0, 0.5)
        oracle.transpose(A, want, perm, size, 1.0, 0.5, dtype="s")
    torch.cuda.synchronize()
    assert_bitexact(dB.cpu().numpy(), want, "150 launches")
    plan.close()


SHIFTED = [([1, 0], [99, 1001]), ([1, 0, 3, 2], [99, 17, 35, 3]), ([1, 0, 2], [45, 77, 9]),
           ([2, 1, 0], [10, 25, 2097]), ([0, 2, 1], [31, 110, 15]), ([2, 0, 1], [23, 13, 240])]


BULK = [([1, 0, 2], [300, 256, 5]), ([2, 0, 1], [8, 64, 1000]), ([1, 0], [1024, 999]), ([3, 1, 0, 2], [16, 20, 24, 9]),
        ([1, 0, 2], [1000, 768, 16])]


@pytest.mark.parametrize("dtype", ["s", "d", "c", "z", "sd", "ds", "zc"])
def test_bulk_a_copies(dtype):
    """A runs moved by one bulk copy each (cp.async.bulk into the stage, an mbarrier per stage):
    bit for bit against the oracle for aligned runs and for shifted runs at A offsets of 0 to 3
    elements, beta = 0 and beta != 0, round-robin and claimed tiles, the shallowest and deepest rings;
    no stage wait runs out of time (run_gpu checks the plan's count)."""
    used = 0
    for perm, size in BULK + SHIFTED:
        for beta in (0.0, -0.5):
            desc = check_case(perm, size, dtype, 1.5, beta, tuning={"bulk_copies": 1})
            used += int((desc.get("tile") or {}).get("bulk", 0))
            for offset in (0, 1, 3):
                check_case(perm, size, dtype, 1.5, beta, offset=offset, tuning={"bulk_copies": 1, "shifted_runs": 1})
            check_case(perm, size, dtype, 1.5, beta, tuning={"bulk_copies": 1, "round_robin": 1, "stages": 3})
            check_case(perm, size, dtype, 1.5, beta, tuning={"bulk_copies": 1, "blocks": 9, "stages": 7,
                                                             "round_robin": -1})
    assert used > 0


LANE_MAPS = [([1, 0, 2, 3], [48, 3, 48, 29]), ([1, 0], [54, 48]), ([2, 3, 1, 0], [17, 22, 53, 12]), ([1, 0], [32, 20]),
             ([1, 2, 0], [18, 31, 58]), ([1, 0], [4, 58]), ([2, 1, 0], [40, 48, 30]), ([1, 2, 3, 0], [29, 54, 59, 29])]


@pytest.mark.parametrize("dtype", ["s", "d", "c", "sd", "ds"])
def test_lane_maps(dtype):
    """Plans whose register path takes B vectors from several B runs per warp (lane_map = 1: maps
    the planner picks against the gather's bank conflicts, in natural or A-sorted run order),
    including maps whose last footprint row reaches past the tile's runs: bit for bit against the
    oracle for beta = 0 and beta != 0, with claimed tiles, bulk copies and round-robin tiles."""
    used = 0
    for perm, size in LANE_MAPS:
        for beta in (0.0, -0.5):
            desc = check_case(perm, size, dtype, 1.5, beta, tuning={"lane_map": 1})
            used += int((desc.get("tile") or {}).get("lane_map", 0) > 0)
            check_case(perm, size, dtype, 1.5, beta, tuning={"lane_map": 1, "round_robin": -1, "blocks": 7})
            check_case(perm, size, dtype, 1.5, beta, tuning={"lane_map": 1, "bulk_copies": 1})
            check_case(perm, size, dtype, 1.5, beta, tuning={"lane_map": 1, "round_robin": 1, "stages": 5})
    assert used > 0


def test_bounded_wait_gives_up_and_the_context_survives():
    """The stage wait of the bulk-copy kernel has a time limit: on a barrier phase that nothing
    completes it gives up after the limit and reports it, and the context stays usable; on a phase
    that completes it does not give up."""
    import ctypes
    import time
    from ttc_b200 import _native
    lib = _native.lib()
    n = ctypes.c_uint(7)
    t0 = time.perf_counter()
    assert lib.ttcb_test_bounded_wait(20_000_000, 0, ctypes.byref(n)) == 0
    assert n.value == 1 and time.perf_counter() - t0 >= 0.02
    assert lib.ttcb_test_bounded_wait(20_000_000, 1, ctypes.byref(n)) == 0
    assert n.value == 0
    check_case([1, 0, 2], [300, 256, 5], "s", 1.5, -0.5, tuning={"bulk_copies": 1})


@pytest.mark.parametrize("dtype", ["s", "d", "c", "sd", "ds", "cz"])
def test_shifted_a_runs(dtype):
    """A runs of odd lengths and offsets copied as the 16-byte chunks that cover them, shifted per
    tile (and by A's own misalignment, offsets of 1 to 3 elements): bit for bit against the oracle,
    for beta = 0 and beta != 0, and equal to the plain layout (shifted_runs = -1)."""
    used = 0
    for perm, size in SHIFTED:
        for beta in (0.0, -0.5):
            for offset in (0, 1, 3):
                desc = check_case(perm, size, dtype, 1.5, beta, offset=offset, tuning={"shifted_runs": 1})
                used += int((desc.get("tile") or {}).get("shifted_runs", 0))
            check_case(perm, size, dtype, 1.5, beta, tuning={"shifted_runs": -1})
            check_case(perm, size, dtype, 1.5, beta, tuning={"shifted_runs": 1, "round_robin": 1, "stages": 5})
            check_case(perm, size, dtype, 1.5, beta, tuning={"shifted_runs": 1, "blocks": 9, "round_robin": -1})
    assert used > 0
