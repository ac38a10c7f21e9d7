"""The multi-GPU policy (replicas only) on two gloo ranks on the CPU: every rank draws its own
seeded problems, the only collective is the max over ranks of the timed region, the job's
throughput counts every rank's bytes over the slowest rank's time, and the reference arm runs on
rank 0 alone."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    from datetime import timedelta
    from pathlib import Path
    import torch
    import torch.distributed as dist
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import ttc_b200.workloads as wl
        from ttc_b200.replicas import job_throughput, max_over_ranks, rank_seed
        cases = wl.sweep_cases(rank_seed(2024, rank))[:4]
        sig = [tuple(c["size"]) + tuple(c["perm"]) for c in cases]
        gathered = [None] * world
        dist.all_gather_object(gathered, sig)
        slowest = max_over_ranks(10.0 + rank)  # rank r "took" 10 + r ms
        thr = job_throughput(1_000_000_000, world, slowest)
        import bench

        class Args:
            pass

        ref_rc = bench.run_reference_arm(Args(), rank, world) if rank != 0 else 0
        out.put((rank, gathered, slowest, thr, ref_rc))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_run_independent_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0, p.exitcode
    results = sorted(q.get() for _ in range(world))
    for rank, gathered, slowest, thr, ref_rc in results:
        assert gathered[0] != gathered[1], "ranks must draw different problems"
        assert slowest == pytest.approx(11.0)
        assert thr == pytest.approx(2e9 / 11e-3 / 1e9)
        assert ref_rc == 0  # ranks other than 0 do no reference work and exit cleanly
