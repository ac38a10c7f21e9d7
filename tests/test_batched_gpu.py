"""Batched mode on the GPU: every problem of a persistent launch (plain and graph-replayed) must equal
the per-call plain kernel and the oracle bit for bit."""
import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, uniform

pytestmark = pytest.mark.gpu


def _problems(seed, count):
    import ttc_b200.workloads as wl
    return wl.batched_cases(seed=seed, count=count, median=4096, lo=64, hi=1 << 16)


@pytest.mark.parametrize("graph", [False, True])
def test_batched_matches_oracle_and_plain_calls(graph):
    import torch
    from ttc_b200 import Plan
    from ttc_b200.batched import Batch
    cases = _problems(5, 300)
    plans, As, Bs, Cs, wants = [], [], [], [], []
    for k, c in enumerate(cases):
        n = int(np.prod(c["size"]))
        a = uniform(n, "s", 100 + k)
        wants.append(oracle.transpose(a, np.zeros(n, np.float32), c["perm"], c["size"], 1.0, 0.0, dtype="s"))
        plans.append(Plan(c["perm"], c["size"], "s"))
        As.append(torch.from_numpy(a).cuda())
        Bs.append(torch.full((n,), float("nan"), device="cuda"))
        Cs.append(torch.full((n,), float("nan"), device="cuda"))
    batch = Batch(plans, As, Bs, alpha=1.0)
    for rep in range(2):  # the second launch re-runs on reset counters
        batch.launch(graph=graph)
    batch.check_status()
    for p, a, cbuf in zip(plans, As, Cs):
        p(a, cbuf, 1.0)
    torch.cuda.synchronize()
    for k, (b, cbuf, w) in enumerate(zip(Bs, Cs, wants)):
        assert_bitexact(b.cpu().numpy(), w, f"batched problem {k} {cases[k]}")
        assert torch.equal(b, cbuf)


def test_batched_beta_mixed_kernels_and_dtypes():
    import torch
    from ttc_b200 import Plan
    from ttc_b200.batched import Batch
    rng = np.random.default_rng(3)
    for dtype in ("d", "zc", "sd"):
        ta, tb = (dtype[0], dtype[1]) if len(dtype) == 2 else (dtype, dtype)
        tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
        plans, As, Bs, wants = [], [], [], []
        for k in range(40):
            r = int(rng.integers(2, 5))
            size = [int(x) for x in rng.integers(1, 40, r)]
            perm = [int(x) for x in rng.permutation(r)]
            n = int(np.prod(size))
            a = uniform(n, ta, k)
            b = uniform(n, tb, 1000 + k)
            alpha, beta = (complex(0.5, -1.0), complex(2.0, 0.25)) if ta in "cz" else (0.5, 2.0)
            wants.append(oracle.transpose(a, b.copy(), perm, size, alpha, beta, dtype=dtype))
            plans.append(Plan(perm, size, dtype, True, tuning={"vec": k % 2}))
            As.append(torch.from_numpy(a).cuda())
            Bs.append(torch.from_numpy(b).cuda())
        Batch(plans, As, Bs, alpha=alpha, beta=beta).launch()
        torch.cuda.synchronize()
        for k, (bb, w) in enumerate(zip(Bs, wants)):
            assert_bitexact(bb.cpu().numpy(), w, f"{dtype} problem {k}")


@pytest.mark.parametrize("dtype", ["s", "d"])
def test_batched_ragged_tiles_and_vector_widths(dtype):
    """Batched problems whose ragged tiles go element-wise inside the batch's ring (ragged = 1), next to
    problems with every access-width pair (full, half and scalar vectors, from the problems' own
    alignment and from vec = 1), small tiles with many tiles per problem, beta = 0 and beta != 0: bit
    for bit against the oracle."""
    import torch
    from ttc_b200 import Plan
    from ttc_b200.batched import Batch
    rng = np.random.default_rng(11)
    tmap = {"s": torch.float32, "d": torch.float64}
    for beta in (0.0, -0.5):
        plans, As, Bs, wants = [], [], [], []
        for k in range(60):
            r = int(rng.integers(2, 5))
            size = [int(x) for x in rng.integers(3, 70, r)]
            if int(np.prod(size)) > 400000:
                size[-1] = 3
            perm = [int(x) for x in rng.permutation(r)]
            n = int(np.prod(size))
            a = uniform(n, dtype, 500 + k)
            b = uniform(n, dtype, 900 + k)
            wants.append(oracle.transpose(a, b.copy(), perm, size, 1.5, beta, dtype=dtype))
            tu = [{"ragged": 1}, {"ragged": 1, "tile_elems": 256}, {"vec": 1}, {}, {"tile_elems": 512}][k % 5]
            plans.append(Plan(perm, size, dtype, beta != 0, tuning=tu))
            As.append(torch.from_numpy(a).cuda())
            Bs.append(torch.from_numpy(b).cuda())
        batch = Batch(plans, As, Bs, alpha=1.5, beta=beta)
        batch.launch()
        batch.check_status()
        torch.cuda.synchronize()
        for k, (bb, w) in enumerate(zip(Bs, wants)):
            assert_bitexact(bb.cpu().numpy(), w, f"{dtype} beta={beta} problem {k}")
        batch.close()


def test_batch_rejects_mixed_types():
    from ttc_b200 import Plan, TTCError
    from ttc_b200.batched import Batch
    import torch
    x = torch.zeros(64, device="cuda", dtype=torch.float64)
    y = torch.zeros(64, device="cuda", dtype=torch.float32)
    with pytest.raises(TTCError):
        Batch([Plan([1, 0], [8, 8], "s"), Plan([1, 0], [8, 8], "d")], [y, x], [y, x])


def test_full_batched_workload_matches_oracle():
    """The batched workload the benchmark times, at full size: 4096 rank-3..5 fp32 problems with
    log-normal element counts (median 64 Ki, 1 Ki..1 Mi), each with the schedule the autotuner's
    measured search picks for it, in one persistent launch replayed from a CUDA graph. Every problem
    is compared bit for bit with the oracle (TTC's reference loop, GPUreference.py:90-137 in the
    TTC project) and with the per-call result of its own plan."""
    import math
    import os
    import torch
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan
    from ttc_b200.autotune import Problem, tune_for_batch
    from ttc_b200.batched import Batch
    cases = wl.batched_cases(seed=7, count=4096)
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev)
    plans, As, Bs, Cs = [], [], [], []
    for k, c in enumerate(cases):
        n = math.prod(c["size"])
        tu = tune_for_batch(Problem(c["perm"], c["size"], "s"), max_impl=6, reps=2) or None
        plans.append(Plan(c["perm"], c["size"], "s", False, tuning=tu))
        gen.manual_seed(1_000_000 + k)
        As.append(torch.rand(n, device=dev, generator=gen).mul_(2).sub_(1))
        Bs.append(torch.full((n,), float("nan"), device=dev))
        Cs.append(torch.full((n,), float("nan"), device=dev))
    batch = Batch(plans, As, Bs, alpha=1.0)
    batch.launch(graph=True)
    batch.launch(graph=True)  # a replay on reset counters
    batch.check_status()
    for p, a, cbuf in zip(plans, As, Cs):
        p(a, cbuf, 1.0, 0.0)
    torch.cuda.synchronize()
    threads = os.cpu_count() or 1
    for k, c in enumerate(cases):
        a = As[k].cpu().numpy()
        want = oracle.transpose(a, np.zeros_like(a), c["perm"], c["size"], 1.0, 0.0, dtype="s", threads=threads)
        assert_bitexact(Bs[k].cpu().numpy(), want, f"batched problem {k} {c} plan={plans[k].describe()}")
        assert torch.equal(Bs[k].view(torch.int32), Cs[k].view(torch.int32)), f"problem {k}: batch vs per-call"
    batch.close()
    for p in plans:
        p.close()
