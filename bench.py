#!/usr/bin/env python3
"""Benchmark of the B200 transposition on the large sweep workload.

A step = one pass over the 64-case sweep: seeded rank-2..6 transpositions with |A| ~ 200 MiB each
(fp32/fp64, half alpha=1/beta=0, half alpha=1.5/beta=-0.5, one extent in [7, 31]), the shapes of TTC's
200 MiB benchmark method. Inputs stay resident in HBM for `value`; `e2e` repeats the metric through
the public call with pinned host buffers and the host<->device copies inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs its own seeded sweep (weak scaling, no collective on the data path);
rank 0 prints one JSON line. `--impl reference` times the reference's CPU implementation of the path
on the host cores (TTC's generated AVX code from oracle/_ref when it was built, otherwise the C port
of TTC's reference loop) on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from ttc_b200.replicas import job_throughput, max_over_ranks, rank_seed  # noqa: E402

METRIC = "transpose GB/s (% of HBM peak); learned-vs-searched plan GB/s and tuning time"
WORKLOAD = ("sweep64: 64 seeded rank-2..6 transpositions, |A|~200 MiB each, fp32/fp64, random "
            "non-identity perms, one extent in [7,31]; even cases alpha=1 beta=0, odd alpha=1.5 beta=-0.5")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--e2e-cases", type=int, default=16)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-sample-cases", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--workload", default="sweep", choices=["sweep", "batched", "case", "configs"],
                    help="sweep: the 64-case 200 MiB sweep (default); batched: 4096 small transpositions "
                         "in one persistent launch against per-call launches; case: one sweep case run "
                         "--reps times with its default plan (a small command for profilers); configs: the "
                         "README shape and the strided mixed-precision shapes, each timed alone")
    ap.add_argument("--schedule", default="learned", choices=["default", "learned"],
                    help="sweep: the planner's default schedule per case, or the learned selector's choice "
                         "(chosen before the timed region: its top-1, timed against the planner default when "
                         "its confidence is low)")
    ap.add_argument("--case", type=int, default=6, help="case: index into the sweep")
    ap.add_argument("--reps", type=int, default=3, help="case: launches")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--batch-tuning", default="search", choices=["search", "default"],
                    help="per-problem schedules: measured search (the autotuner) or the planner default")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str | None):
        self.device_id = device_id
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.device_id:
            cmd += ["-i", self.device_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def device_uuid(dev):
    """nvidia-smi's id of a torch device (its UUID), so the sampler reads this GPU only."""
    import torch
    uuid = getattr(torch.cuda.get_device_properties(dev), "uuid", None)
    return f"GPU-{uuid}" if uuid is not None else None


def measured_peak_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic_per_gb(kernel: str):
    """DRAM bytes per algorithmic byte of the dominant kernel, from the committed ncu summary."""
    f = ROOT / "profiles" / f"{kernel}_sweep_traffic.md"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_algorithmic_byte:\s*([0-9.]+)", f.read_text())
    return float(m.group(1)) if m else None


# ------------------------------------------------------------------------------------------------
def cpu_prepare(cases):
    """Seeded host inputs for the CPU baseline sample (untimed), 64-byte aligned."""
    from oracle.cpu_ref import aligned
    out = []
    for c in cases:
        real = np.float32 if c["dtype"] == "s" else np.float64
        na = math.prod(c["size"])
        A = aligned(na, real)
        B = aligned(na, real)
        A[:] = np.random.default_rng(c["seed"]).uniform(-1, 1, na)
        B[:] = np.random.default_rng(c["seed"] + 1).uniform(-1, 1, na)
        out.append((c, A, B))
    return out


def cpu_reference_run(prepared, threads, min_seconds=10.0, max_passes=50):
    """Times the reference's CPU implementation on a bounded sample; returns (GB/s, kind, desc)."""
    import oracle
    from oracle import cpu_ref
    import ttc_b200.workloads as wl
    impl = cpu_ref.available()
    if impl is not None and not all(cpu_ref._key(c) in impl.keys for c, _, _ in prepared):
        impl = None
    kind = "reference" if impl else "port"
    total_bytes, total_time = 0, 0.0
    t_start = time.perf_counter()
    passes = 0
    while True:
        for c, A, B in prepared:
            t0 = time.perf_counter()
            if impl:
                impl(c, A, B, threads)
            else:
                oracle.transpose(A, B, c["perm"], c["size"], c["alpha"], c["beta"], dtype=c["dtype"],
                                 threads=threads)
            total_time += time.perf_counter() - t0
            total_bytes += wl.case_bytes(c)
        passes += 1
        if time.perf_counter() - t_start >= min_seconds or passes >= max_passes:
            break
    per_pass = sum(wl.case_bytes(c) for c, _, _ in prepared)
    desc = (f"first {len(prepared)} sweep cases ({per_pass / 1e9:.2f} GB per pass) x {passes} passes, "
            f"{threads} threads, " + ("TTC's generated AVX code (best variant of TTC's own search)"
                                       if impl else "C port of TTC's OpenMP reference loop"))
    return total_bytes / total_time / 1e9, kind, desc


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    import ttc_b200.workloads as wl
    threads = os.cpu_count() or 1
    cases = wl.sweep_cases(args.seed)[: max(1, args.cpu_sample_cases)]
    prepared = cpu_prepare(cases)
    for _ in range(args.warmup):
        cpu_reference_run(prepared[:1], threads, min_seconds=0.0, max_passes=1)
    t0 = time.perf_counter()
    vals = []
    for _ in range(args.steps):
        v, kind, desc = cpu_reference_run(prepared, threads, min_seconds=0.0, max_passes=1)
        vals.append(v)
    wall = time.perf_counter() - t0
    value = statistics.median(vals)
    total_bytes = sum(wl.case_bytes(c) for c in cases)
    line = {"metric": METRIC, "value": round(value, 3), "unit": "GB/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(wall / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded uniform[-1,1])",
            "config": {"workload": WORKLOAD, "sample_cases": len(cases), "bytes_per_step": total_bytes},
            "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": kind,
                             "sample": desc + f"; median of {args.steps} steps"},
            "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.workload == "batched":
        return run_batched(args, rank, world, local)
    if args.workload == "case":
        return run_case(args)
    if args.workload == "configs":
        return run_configs(args)

    import torch
    import torch.distributed as dist
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    cases = wl.sweep_cases(rank_seed(args.seed, rank))[: args.cases]
    tmap = {"s": torch.float32, "d": torch.float64}

    # resident inputs, seeded on the device
    gen = torch.Generator(device=dev)
    items = []
    for c in cases:
        n = math.prod(c["size"])
        gen.manual_seed(c["seed"])
        A = torch.rand(n, dtype=tmap[c["dtype"]], device=dev, generator=gen).mul_(2).sub_(1)
        gen.manual_seed(c["seed"] + 1)
        B = torch.rand(n, dtype=tmap[c["dtype"]], device=dev, generator=gen).mul_(2).sub_(1)
        tuning = None
        if args.schedule == "learned":
            from ttc_b200 import cost_model
            from ttc_b200.autotune import Problem
            # the network's top-1; below its confidence threshold the top-1 and the planner default
            # are timed (outside the timed region) and the faster one is kept
            sel = cost_model.select(Problem(c["perm"], c["size"], c["dtype"], c["alpha"], c["beta"]),
                                    verify=False, measure_choice=False)
            if sel["results"]:
                tuning = min(sel["results"], key=lambda r: r.time_ms).tuning or None
            else:
                tuning = sel["candidates"][int(sel["order"][0])][0] or None
        plan = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning=tuning)
        items.append((c, plan, A, B))
    torch.cuda.synchronize()
    bytes_per_step = sum(p.bytes for _, p, _, _ in items)
    stream = torch.cuda.current_stream()

    def step(events=None):
        for k, (c, plan, A, B) in enumerate(items):
            if events is not None:
                events[k][0].record(stream)
            plan(A, B, c["alpha"], c["beta"], stream)
            if events is not None:
                events[k][1].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(device_uuid(dev)).start()
    time.sleep(0.3)
    evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in items]
           for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for s in range(args.steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    # a second pass, timed per launch, splits the device time by kernel for the roofline (events
    # between launches would break the overlap of consecutive launches, so `value` comes from the
    # pass above, which has none)
    for s in range(args.steps):
        step(evs[s])
    torch.cuda.synchronize()
    elapsed_ms = max_over_ranks(t0.elapsed_time(t1), dev)
    ms_per_step = elapsed_ms / args.steps
    value = job_throughput(bytes_per_step, world, ms_per_step)

    # per-kernel split of device time (dominant kernel -> roofline)
    kinds = [p.describe()["kernel"] for _, p, _, _ in items]
    # a staged tile plan with ragged tiles also launches its edge plans (or the ragged-tile kernel)
    launches_per_step = sum(p.launches() for _, p, _, _ in items)
    per_kind = {}
    for s in range(args.steps):
        for k, (c, plan, A, B) in enumerate(items):
            ms = evs[s][k][0].elapsed_time(evs[s][k][1])
            d = per_kind.setdefault(kinds[k], [0.0, 0, 0])
            d[0] += ms
            d[1] += plan.bytes
            d[2] += 1
    dom = max(per_kind, key=lambda k: per_kind[k][0])
    dom_ms, dom_bytes, dom_n = per_kind[dom]
    peak, peak_src = measured_peak_gbs()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    tr = ncu_traffic_per_gb(f"{dom}_kernel")
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_source": peak_src,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "kernel": f"{dom}_kernel",
                "launches": dom_n, "algorithmic_bytes_per_launch": int(dom_bytes / dom_n),
                "traffic": (int(tr * dom_bytes / dom_n) if tr else None),
                "split": {k: {"ms": round(v[0], 3), "GBps": round(v[1] / (v[0] / 1e3) / 1e9, 1), "launches": v[2]}
                          for k, v in per_kind.items()}}

    # end to end through the public call with pinned host buffers
    e2e = run_e2e(args, items, stream, dev, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            prepared = cpu_prepare(cases[: max(1, args.cpu_sample_cases)])
            v, kind, desc = cpu_reference_run(prepared, os.cpu_count() or 1, min_seconds=10.0)
            cpu = {"value": round(v, 3), "unit": "GB/s", "cores": os.cpu_count() or 1, "kind": kind, "sample": desc}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GB/s", "cores": os.cpu_count() or 1, "kind": "port",
                   "sample": f"failed: {ex}"}

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded uniform[-1,1])",
                "pct_of_hbm_peak": round(100 * value / world / peak, 2),
                "config": {"workload": WORKLOAD, "cases": len(items), "bytes_per_step_per_gpu": bytes_per_step,
                           "schedules": ("learned selector (top-1; timed against the planner default when its confidence "
                                         "< 0.1)" if args.schedule == "learned" else "planner default"),
                           "l2": "inputs larger than L2 (|A| ~ 200 MiB per case); no flush needed",
                           "parallelism": f"replicas x{world} (independent seeded sweeps, no collective)"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
                "gpu_launches": launches_per_step * args.steps}
        print(json.dumps(line), flush=True)
    for _, p, _, _ in items:
        p.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def parse_cpulist(text: str) -> set:
    """CPU numbers of a Linux cpulist ("0-3,8,10-11")."""
    cpus = set()
    for part in text.strip().split(","):
        if part:
            lo, _, hi = part.partition("-")
            cpus.update(range(int(lo), int(hi or lo) + 1))
    return cpus


class GpuLocalCpus:
    """Runs its body on the CPUs of the GPU's own NUMA node (from the PCI device's `local_cpulist`),
    so that pinned host buffers allocated there are first touched, and placed, on the memory next to
    the GPU's PCIe root; the process's previous CPU set is restored afterwards. A no-op where the
    node is not known."""

    def __init__(self, dev):
        self.dev, self.old = dev, None

    def __enter__(self):
        import torch
        try:
            pr = torch.cuda.get_device_properties(self.dev)
            path = Path(f"/sys/bus/pci/devices/{pr.pci_domain_id:04x}:{pr.pci_bus_id:02x}:"
                        f"{pr.pci_device_id:02x}.0/local_cpulist")
            cpus = parse_cpulist(path.read_text())
            old = os.sched_getaffinity(0)
            use = cpus & old
            if use and use != old:
                os.sched_setaffinity(0, use)
                self.old = old
        except (OSError, ValueError, AttributeError, RuntimeError):
            self.old = None
        return self

    def __exit__(self, *exc):
        if self.old is not None:
            os.sched_setaffinity(0, self.old)
        return False


def run_e2e(args, items, stream, dev, world):
    """The metric through the public call from pinned host buffers: per case, A (and B when
    beta != 0) is copied in, transposed and B copied out. Copies in and out run on their own
    streams so that PCIe carries both directions at once (case i+1 comes in while case i goes out);
    each case's copy-in, kernel and copy-out are ordered by events."""
    import torch
    sub = items[: max(1, min(args.e2e_cases, len(items)))]
    host = []
    with GpuLocalCpus(dev):  # pinned buffers on the host memory next to the GPU
        for c, plan, A, B in sub:
            hA = torch.empty(A.numel(), dtype=A.dtype, pin_memory=True)
            hB = torch.empty(B.numel(), dtype=B.dtype, pin_memory=True)
            hA.copy_(A)
            hB.copy_(B)
            host.append((hA, hB))
        outs = [torch.empty_like(hB, pin_memory=True) for _, hB in host]
    h2d = sum(hA.numel() * hA.element_size() + (hB.numel() * hB.element_size() if c["beta"] != 0 else 0)
              for (c, _, _, _), (hA, hB) in zip(sub, host))
    d2h = sum(hB.numel() * hB.element_size() for _, hB in host)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    out_done = [None] * len(sub)  # per case: its last copy-out, before its buffers are refilled

    def one():
        for k, ((c, plan, A, B), (hA, hB), o) in enumerate(zip(sub, host, outs)):
            with torch.cuda.stream(s_in):
                if out_done[k] is not None:
                    s_in.wait_event(out_done[k])
                A.copy_(hA, non_blocking=True)
                if c["beta"] != 0:
                    B.copy_(hB, non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(s_in)
            stream.wait_event(ev_in)
            plan(A, B, c["alpha"], c["beta"], stream)
            ev_k = torch.cuda.Event()
            ev_k.record(stream)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_k)
                o.copy_(B, non_blocking=True)
                out_done[k] = torch.cuda.Event()
                out_done[k].record(s_out)
        stream.wait_stream(s_out)

    one()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    s_in.wait_stream(stream)
    s_out.wait_stream(stream)
    for _ in range(args.e2e_steps):
        one()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1) / args.e2e_steps, dev)
    nbytes = sum(p.bytes for _, p, _, _ in sub)
    return {"value": round(nbytes * world / (ms / 1e3) / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "cases": len(sub), "ms_per_step": round(ms, 3),
            "note": ("pinned host A (and B when beta != 0) copied in and B copied out for every case inside the "
                     "timed region; copy-in and copy-out on separate streams (PCIe both directions)")}


def run_configs(args):
    """The single-problem configurations: TTC's README shape (perm 1,0,2 / 1000,768,16, fp32,
    alpha = beta = 1) and the strided mixed-precision shape (perm 3,1,0,2 / 96,80,72,64, lda + 8,0,4,0;
    z->c with alpha = (0.5, 0.25) and d->s with alpha = 0.5, beta = 0). Inputs uniform[-1,1] from the
    seed (B from seed + 1), resident; the L2 is flushed (2x its size written) before every timed
    launch; CUDA events, `--steps` launches after `--warmup`. Prints one JSON line."""
    import torch
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan
    tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
    flush = torch.empty(2 * 126 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = []
    for name, c in [("readme_1000x768x16_s_beta1", wl.readme_case())] + \
                   [(f"strided_96x80x72x64_{c['dtype']}", c) for c in wl.strided_cases()]:
        ta, tb = (c["dtype"][0], c["dtype"][1]) if len(c["dtype"]) == 2 else (c["dtype"], c["dtype"])
        lda = c.get("lda") or c["size"]
        na = math.prod(lda[:-1]) * c["size"][-1]
        nb = math.prod(c["size"])
        gen = torch.Generator(device="cuda")
        gen.manual_seed(args.seed)
        A = (torch.rand(na, dtype=tmap[ta], device="cuda", generator=gen) * 2 - 1)
        gen.manual_seed(args.seed + 1)
        B = (torch.rand(nb, dtype=tmap[tb], device="cuda", generator=gen) * 2 - 1)
        plan = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, lda=c.get("lda"))
        for _ in range(args.warmup):
            plan(A, B, c["alpha"], c["beta"])
        ms = []
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            plan(A, B, c["alpha"], c["beta"])
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        med = statistics.median(ms)
        peak, src = measured_peak_gbs()
        d = plan.describe()
        out.append({"config": name, "perm": c["perm"], "size": c["size"], "lda": c.get("lda"), "dtype": c["dtype"],
                    "alpha": str(c["alpha"]), "beta": c["beta"], "bytes": plan.bytes,
                    "GBps_median": round(plan.bytes / (med / 1e3) / 1e9, 1),
                    "GBps_best": round(plan.bytes / (min(ms) / 1e3) / 1e9, 1),
                    "pct_of_hbm_peak": round(100 * plan.bytes / (med / 1e3) / 1e9 / peak, 1),
                    "kernel": d["kernel"], "tile": d.get("tile"), "vec": [d["vecA"], d["vecB"]]})
        plan.close()
    print(json.dumps({"workload": "configs", "steps": args.steps, "warmup": args.warmup, "l2": "flushed",
                      "results": out}), flush=True)
    return 0


def run_case(args):
    """One sweep case, `--reps` launches of its default plan on seeded resident inputs; prints the
    plan and the mean GB/s (CUDA events). Meant to sit under a profiler."""
    import torch
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan
    c = wl.sweep_cases(args.seed)[args.case]
    tmap = {"s": torch.float32, "d": torch.float64}
    n = math.prod(c["size"])
    gen = torch.Generator(device="cuda")
    gen.manual_seed(c["seed"])
    A = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen)
    B = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen)
    plan = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.reps):
        plan(A, B, c["alpha"], c["beta"])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.reps, 1)
    print(json.dumps({"case": args.case, "perm": c["perm"], "size": c["size"], "dtype": c["dtype"],
                      "beta": c["beta"], "GBps": round(plan.bytes / (ms / 1e3) / 1e9, 1), "bytes": plan.bytes,
                      "plan": plan.describe()}), flush=True)
    plan.close()
    return 0


# ------------------------------------------------------------------------------------------------
BATCH_WORKLOAD = ("batched4096: seeded rank-3..5 fp32 transpositions, random perms, element counts "
                  "log-normal median 64Ki clipped to [1Ki, 1Mi], alpha=1 beta=0")


def run_batched(args, rank, world, local):
    """Batched mode: every problem of the batch in one persistent launch (plain and replayed from a
    captured CUDA graph) against the same problems launched one call at a time: a Python loop over
    the public call, that loop captured into a CUDA graph, and a loop that synchronizes after every
    call as TTC's generated wrapper does. Every batched result is compared bit for bit with the
    per-call result."""
    import torch
    import torch.distributed as dist
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan
    from ttc_b200.autotune import Bench, Problem, tune_for_batch
    from ttc_b200.batched import Batch

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    cases = wl.batched_cases(seed=rank_seed(7, rank), count=args.batch_count)
    t_tune = time.perf_counter()
    plans, As, Bs, Cs = [], [], [], []
    gen = torch.Generator(device=dev)
    for k, c in enumerate(cases):
        n = math.prod(c["size"])
        tu = None
        if args.batch_tuning == "search":
            tu = tune_for_batch(Problem(c["perm"], c["size"], "s"), max_impl=6, reps=2) or None
        plans.append(Plan(c["perm"], c["size"], "s", False, tuning=tu))
        gen.manual_seed(1_000_000 + k)
        As.append(torch.rand(n, device=dev, generator=gen).mul_(2).sub_(1))
        Bs.append(torch.full((n,), float("nan"), device=dev))
        Cs.append(torch.full((n,), float("nan"), device=dev))
    t_tune = time.perf_counter() - t_tune
    batch = Batch(plans, As, Bs, alpha=1.0)
    total = batch.bytes
    stream = torch.cuda.current_stream()

    def timed(fn, steps):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / steps, dev)

    def per_call():
        for p, a, cbuf in zip(plans, As, Cs):
            p(a, cbuf, 1.0, 0.0, stream)

    def per_call_sync():
        for p, a, cbuf in zip(plans, As, Cs):
            p(a, cbuf, 1.0, 0.0, stream)
            torch.cuda.synchronize()

    for _ in range(args.warmup):
        batch.launch(stream)
        batch.launch(stream, graph=True)
        per_call()
    batch.check_status(stream)
    g = torch.cuda.CUDAGraph()
    s2 = torch.cuda.Stream()
    s2.wait_stream(stream)
    with torch.cuda.stream(s2):
        with torch.cuda.graph(g, stream=s2):
            for p, a, cbuf in zip(plans, As, Cs):
                p(a, cbuf, 1.0, 0.0, s2)
    stream.wait_stream(s2)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()

    sampler = ClockSampler(device_uuid(dev)).start()
    time.sleep(0.3)
    ms_graph = timed(lambda: batch.launch(stream, graph=True), args.steps)
    clocks = sampler.stop()
    ms_plain = timed(lambda: batch.launch(stream), args.steps)
    ms_calls = timed(per_call, max(1, args.steps // 2))
    ms_calls_graph = timed(g.replay, args.steps)
    ms_calls_sync = timed(per_call_sync, 1)
    batch.check_status(stream)

    # every batched result against the per-call result, bit for bit
    per_call()
    torch.cuda.synchronize()
    mismatches = sum(0 if torch.equal(b.view(torch.int32), cbuf.view(torch.int32)) else 1 for b, cbuf in zip(Bs, Cs))
    gbs = lambda ms: round(total * world / (ms / 1e3) / 1e9, 2)
    kinds = {}
    for p in plans:
        k = p.describe()["kernel"]
        kinds[k] = kinds.get(k, 0) + 1
    if rank == 0:
        line = {"metric": "batched transpose GB/s (one persistent launch under a CUDA graph)",
                "value": gbs(ms_graph), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms_graph, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (seeded uniform[-1,1])",
                "config": {"workload": BATCH_WORKLOAD, "problems": len(cases), "bytes_per_step_per_gpu": total,
                           "schedules": ("measured search per problem over tile shape x raster order "
                                         "(staged kernel, 6 candidates, 2 reps)"
                                         if args.batch_tuning == "search" else "planner default"),
                           "tuning_seconds": round(t_tune, 1), "plan_kinds": kinds,
                           "l2": f"{total / 1e9:.2f} GB per step, larger than L2"},
                "batched_plain_launch": {"GBps": gbs(ms_plain), "ms": round(ms_plain, 4)},
                "per_call": {"python_loop": {"GBps": gbs(ms_calls), "ms": round(ms_calls, 3)},
                             "graph_of_calls": {"GBps": gbs(ms_calls_graph), "ms": round(ms_calls_graph, 3)},
                             "sync_each_call": {"GBps": gbs(ms_calls_sync), "ms": round(ms_calls_sync, 3)}},
                "speedup": {"vs_python_loop": round(ms_calls / ms_graph, 2),
                            "vs_graph_of_calls": round(ms_calls_graph / ms_graph, 2),
                            "vs_sync_each_call": round(ms_calls_sync / ms_graph, 2)},
                "check": {"problems": len(cases), "mismatches_vs_per_call": mismatches},
                "clocks": clocks, "gpu_launches": args.steps}
        print(json.dumps(line), flush=True)
    del g
    batch.close()
    for p in plans:
        p.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 1 if mismatches else 0


if __name__ == "__main__":
    sys.exit(main())
