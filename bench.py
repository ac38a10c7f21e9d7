#!/usr/bin/env python3
"""Benchmark of the B200 transposition on the large sweep workload.

A step = one pass over the 64-case sweep: seeded rank-2..6 transpositions with |A| ~ 200 MiB each
(fp32/fp64, half alpha=1/beta=0, half alpha=1.5/beta=-0.5, one extent in [7, 31]), the shapes of TTC's
200 MiB benchmark method. Inputs stay resident in HBM for `value`; `e2e` repeats the metric over the
same 64 cases through the public call with pinned host buffers and the host<->device copies inside
the timed region, beside the PCIe bandwidth measured in the same run. The CPU baseline (TTC's own
generated AVX code, rebuilt for this host with TTC's Makefile flags) runs the same 64 cases.
Each case is timed with the schedule that a measured search picked for it before the timed region
(TTC's method: every candidate timed and checked against the first); `schedule_kinds` gives the sweep
under the planner's defaults and the learned selector's choices too, with each one's tuning time.
On one GPU the line also carries the other configurations: the README shape, the strided mixed-
precision shapes, the batched workload against per-call launches, and the learned selector against
a fresh measured search on held-out problems.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-extras]

Under torchrun every rank runs its own seeded sweep (weak scaling, no collective on the data path);
rank 0 prints one JSON line. `--impl reference` times the reference's CPU implementation of the path
on the host cores (TTC's generated AVX code from oracle/_ref, rebuilt for the host; the C port of
TTC's reference loop where it was not built) on rank 0 only, over the same 64 cases.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
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
L2_NOTE = "inputs larger than L2 (|A| ~ 200 MiB per case); no flush needed"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline: minimum seconds of timed passes")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations (README, strided, batched, selector) in the sweep line")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--workload", default="sweep", choices=["sweep", "batched", "case", "configs", "batchcase"],
                    help="sweep: the 64-case 200 MiB sweep (default); batched: 4096 small transpositions "
                         "in one persistent launch against per-call launches; case: one sweep case run "
                         "--reps times with its default plan (a small command for profilers); configs: the "
                         "README shape and the strided mixed-precision shapes, each timed alone; batchcase: the "
                         "batched workload with the planner's schedules launched --reps times (for profilers)")
    ap.add_argument("--schedule", default="search", choices=["search", "learned", "default"],
                    help="sweep: the schedule each case is timed with, chosen before the timed region. "
                         "search: TTC's method, every candidate schedule (up to --search-candidates) timed "
                         "and checked bit for bit against the first, the fastest kept; learned: the learned "
                         "selector (its top-1 on a large predicted gain over the planner default, the "
                         "fastest of its top candidates and the default, timed, on a moderate one); "
                         "default: the planner's. Unless --no-extras, the other two are timed as well and "
                         "reported beside it")
    ap.add_argument("--search-candidates", type=int, default=200,
                    help="sweep: candidate schedules per case for the measured search (TTC's default "
                         "maxImplementations; the sweep's cases have 1 to 112 candidates, 49 on average)")
    ap.add_argument("--case", type=int, default=6, help="case: index into the sweep")
    ap.add_argument("--reps", type=int, default=3, help="case / batchcase: launches")
    ap.add_argument("--tuning", default=None, help="case: a schedule (JSON of ttcb_tuning fields) instead of the "
                                                   "planner's default")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--batch-tuning", default="default", choices=["search", "default"],
                    help="per-problem schedules: the planner default (measured faster on the 4096-problem batch, "
                         "1764 against 1699 GB/s, and repeatable) or a short measured search per problem")
    ap.add_argument("--selector-cases", type=int, default=40,
                    help="held-out problems for the learned selector's fresh head to head")
    return ap.parse_args(argv)


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


def kernel_name(desc: dict) -> str:
    """The kernel that moves (almost) all of a plan's elements on its default path."""
    if desc["kernel"] == "row":
        return "row_kernel"
    t = desc.get("tile") or {}
    v = desc.get("tile_variant", 0)
    if t.get("async") and v in (0, 3):
        return "tile_async_kernel"
    return "tile_fast_kernel" if (v == 2 or (v == 0 and t.get("fast"))) else "tile_kernel"


def sweep_config(cases: int, bytes_per_step: int, world: int) -> dict:
    """The `config` of the sweep line; both arms print the same one."""
    return {"workload": WORKLOAD, "cases": cases, "bytes_per_step_per_gpu": bytes_per_step, "l2": L2_NOTE,
            "parallelism": f"replicas x{world} (independent seeded sweeps, no collective)"}


# ------------------------------------------------------------------------------------------------
# CPU baseline: the reference's own CPU implementation of the path on this host's cores
def host_inputs(cases, threads):
    """Seeded 32-byte aligned host inputs (A uniform[-1,1) from the case seed, B from seed + 1) for
    the reference arm, filled in parallel."""
    from oracle.cpu_ref import aligned

    def one(c):
        real = np.float32 if c["dtype"] == "s" else np.float64
        n = math.prod(c["size"])
        A, B = aligned(n, real), aligned(n, real)
        A[:] = np.random.default_rng(c["seed"]).uniform(-1, 1, n)
        B[:] = np.random.default_rng(c["seed"] + 1).uniform(-1, 1, n)
        return c, A, B

    with cf.ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        return list(ex.map(one, cases))


class CpuReference:
    """TTC's generated AVX code for every case it was built for (rebuilt for this host with TTC's own
    Makefile flags), and the C port of TTC's reference loop for any case it was not."""

    def __init__(self, cases):
        from oracle import cpu_ref
        self.note = ""
        try:
            impl = cpu_ref.available(native=True)
        except Exception as ex:  # a failed host build falls back to the portable build
            impl = cpu_ref.available()
            self.note = f"; host build failed ({type(ex).__name__}), portable build used"
        self.impl = impl
        self.covered = sum(1 for c in cases if impl is not None and cpu_ref._key(c) in impl.keys)
        self.total = len(cases)
        self.kind = "reference" if self.covered else "port"

    def run(self, c, A, B, threads):
        import oracle
        from oracle import cpu_ref
        if self.impl is not None and cpu_ref._key(c) in self.impl.keys:
            self.impl(c, A, B, threads)
        else:
            oracle.transpose(A, B, c["perm"], c["size"], c["alpha"], c["beta"], dtype=c["dtype"], threads=threads)

    def describe(self, threads) -> str:
        if not self.covered:
            return f"C port of TTC's OpenMP reference loop, {threads} threads" + self.note
        i = self.impl
        s = (f"TTC's generated AVX code, the variant TTC's own search picked per case (--maxImplementations="
             f"{i.max_implementations}, searched on a {i.threads_at_tuning}-thread build host), compiled on this "
             f"host with {i.flags} (compile {i.compile_seconds:.0f} s, outside the timing), {threads} threads")
        if self.covered < self.total:
            s += f"; {self.total - self.covered} of {self.total} cases by the C port of TTC's reference loop"
        return s + self.note


def cpu_passes(ref: CpuReference, prepared, threads, min_seconds=0.0, max_passes=1):
    """Timed passes over every prepared case; returns (GB/s, passes, seconds)."""
    import ttc_b200.workloads as wl
    per_pass = sum(wl.case_bytes(c) for c, _, _ in prepared)
    total_t, passes = 0.0, 0
    while True:
        t0 = time.perf_counter()
        for c, A, B in prepared:
            ref.run(c, A, B, threads)
        total_t += time.perf_counter() - t0
        passes += 1
        if total_t >= min_seconds or passes >= max_passes:
            break
    return per_pass * passes / total_t / 1e9, passes, total_t


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    import ttc_b200.workloads as wl
    threads = os.cpu_count() or 1
    cases = wl.sweep_cases(args.seed)[: args.cases]
    ref = CpuReference(cases)
    prepared = host_inputs(cases, threads)
    for _ in range(args.warmup):
        cpu_passes(ref, prepared, threads)
    vals, t_all = [], 0.0
    for _ in range(args.steps):
        v, _, t = cpu_passes(ref, prepared, threads)
        vals.append(v)
        t_all += t
    value = statistics.median(vals)
    total_bytes = sum(wl.case_bytes(c) for c in cases)
    desc = ref.describe(threads) + f"; all {len(cases)} sweep cases per step, median of {args.steps} steps"
    line = {"metric": METRIC, "value": round(value, 3), "unit": "GB/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_all / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded uniform[-1,1])", "config": sweep_config(len(cases), total_bytes, 1),
            "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": ref.kind,
                             "sample": desc},
            "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
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


def measure_pcie(dev, nbytes=1 << 30, reps=3):
    """Pinned host<->device copy bandwidth of this GPU's link: each direction alone and both at once
    (GB/s, best of `reps`, CUDA events)."""
    import torch
    with GpuLocalCpus(dev):
        h_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        h_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_in = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d_out = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(fn):
        best = float("inf")
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            cur = torch.cuda.current_stream()
            e0.record(cur)
            s1.wait_stream(cur)
            s2.wait_stream(cur)
            fn()
            cur.wait_stream(s1)
            cur.wait_stream(s2)
            e1.record(cur)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    def h2d():
        with torch.cuda.stream(s1):
            d_in.copy_(h_in, non_blocking=True)

    def d2h():
        with torch.cuda.stream(s2):
            h_out.copy_(d_out, non_blocking=True)

    def both():
        h2d()
        d2h()

    h2d(), d2h()
    t_in, t_out, t_both = timed(h2d), timed(d2h), timed(both)
    gb = nbytes / 1e9
    out = {"h2d_gbs": round(gb / (t_in / 1e3), 2), "d2h_gbs": round(gb / (t_out / 1e3), 2),
           "duplex_gbs_each_way": round(gb / (t_both / 1e3), 2), "bytes": nbytes}
    del h_in, h_out, d_in, d_out
    return out


def run_e2e(args, items, stream, dev, world, pcie):
    """The metric through the public call from pinned host buffers, over every case of the sweep:
    per case, A (and B when beta != 0) is copied in, transposed and B copied out. Copies in and out
    run on their own streams so that PCIe carries both directions at once (case i+1 comes in while
    case i goes out); each case's copy-in, kernel and copy-out are ordered by events. Results go to a
    ring of four pinned output buffers. Returns (e2e dict, per-case host buffers)."""
    import torch
    host = []
    with GpuLocalCpus(dev):  # pinned buffers on the host memory next to the GPU
        for c, plan, A, B in items:
            hA = torch.empty(A.numel(), dtype=A.dtype, pin_memory=True)
            hA.copy_(A)
            hB = None
            if c["beta"] != 0:
                hB = torch.empty(B.numel(), dtype=B.dtype, pin_memory=True)
                hB.copy_(B)
            host.append((hA, hB))
        big = max(B.numel() * B.element_size() for _, _, _, B in items)
        ring = [torch.empty(big, dtype=torch.uint8, pin_memory=True) for _ in range(4)]
    h2d = sum(hA.numel() * hA.element_size() + (hB.numel() * hB.element_size() if hB is not None else 0)
              for hA, hB in host)
    d2h = sum(B.numel() * B.element_size() for _, _, _, B in items)
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    out_done = [None] * len(items)  # per case: its last copy-out, before its device buffers are refilled
    ring_done = [None] * len(ring)  # per ring slot: its last copy-out

    def one():
        for k, ((c, plan, A, B), (hA, hB)) in enumerate(zip(items, host)):
            with torch.cuda.stream(s_in):
                if out_done[k] is not None:
                    s_in.wait_event(out_done[k])
                A.copy_(hA, non_blocking=True)
                if hB is not None:
                    B.copy_(hB, non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(s_in)
            stream.wait_event(ev_in)
            plan(A, B, c["alpha"], c["beta"], stream)
            ev_k = torch.cuda.Event()
            ev_k.record(stream)
            slot = k % len(ring)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_k)
                nb = B.numel() * B.element_size()
                ring[slot][:nb].copy_(B.view(torch.uint8), non_blocking=True)
                out_done[k] = torch.cuda.Event()
                out_done[k].record(s_out)
                ring_done[slot] = out_done[k]
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
    nbytes = sum(p.bytes for _, p, _, _ in items)
    out = {"value": round(nbytes * world / (ms / 1e3) / 1e9, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "cases": len(items), "ms_per_step": round(ms, 3),
           "note": ("pinned host A (and B when beta != 0) copied in and B copied out for every case inside the "
                    "timed region; copy-in and copy-out on separate streams (PCIe both directions)")}
    if pcie:
        # the fastest the copies alone could go on this link: each direction at the rate it reaches while
        # the other direction is busy (a lower bound on time, so an upper bound on e2e GB/s)
        duplex = pcie["duplex_gbs_each_way"]
        t_min = max(h2d, d2h) / (duplex * 1e9)
        bound = nbytes / t_min / 1e9
        out["pcie"] = pcie
        out["pcie_bound_gbs"] = round(bound, 2)
        out["frac_of_pcie_bound"] = round(out["value"] / world / bound, 4)
    del ring
    return out, host


def cpu_baseline_on(items, host, threads, min_seconds):
    """TTC's generated code over every sweep case, on the pinned host copies of the GPU inputs
    (A; B where beta != 0, else a shared scratch buffer the code only writes)."""
    cases = [c for c, _, _, _ in items]
    ref = CpuReference(cases)
    from oracle.cpu_ref import aligned
    out_bytes = max([hA.numel() * hA.element_size() for hA, hB in host if hB is None] or [0])
    scratch = aligned(max(out_bytes, 64), np.uint8)  # B of the beta == 0 cases: written, never read
    prepared = []
    for (c, _, _, _), (hA, hB) in zip(items, host):
        a = hA.numpy()
        b = hB.numpy() if hB is not None else scratch[: a.nbytes].view(a.dtype)
        if a.ctypes.data % 32 or b.ctypes.data % 32:  # TTC's aligned vector accesses need 32 bytes
            a2, b2 = aligned(a.size, a.dtype), aligned(b.size, b.dtype)
            a2[:], b2[:] = a, b
            a, b = a2, b2
        prepared.append((c, a, b))
    cpu_passes(ref, prepared, threads)  # warm-up pass
    v, passes, secs = cpu_passes(ref, prepared, threads, min_seconds=min_seconds, max_passes=1000)
    return {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": ref.kind,
            "sample": (ref.describe(threads) + f"; all {len(prepared)} sweep cases per pass, {passes} passes in "
                       f"{secs:.1f} s, on the same data as the GPU run")}


# ------------------------------------------------------------------------------------------------
def run_sweep(args, rank, world, local):
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

    # the learned selector needs its trained model; without one the planner's defaults are timed
    # and the line says so
    schedule_note = None
    learned_ok = True
    try:
        from ttc_b200 import cost_model
        cost_model.load_default()
    except Exception as ex:
        learned_ok = False
        if args.schedule == "learned":
            args.schedule = "default"
            schedule_note = f"learned model unavailable ({type(ex).__name__}: {ex}); planner defaults timed"
    # the headline's schedules first, then (unless --no-extras) the other kinds for the comparison
    sched_kinds = [args.schedule] + ([k for k in ("default", "learned", "search")
                                if k != args.schedule and (k != "learned" or learned_ok)]
                               if not args.no_extras else [])

    def choose(kind, c):
        from ttc_b200.autotune import Problem, search
        p = Problem(c["perm"], c["size"], c["dtype"], c["alpha"], c["beta"])
        if kind == "learned":
            return cost_model.choose_tuning(p)
        if kind == "search":
            r = search(p, max_impl=args.search_candidates, reps=3, verify=True, seed=c["seed"])
            torch.cuda.empty_cache()
            return dict(r["best"].tuning) or None
        return None

    # resident inputs, seeded on the device
    gen = torch.Generator(device=dev)
    items = []
    tunings = {k: [] for k in sched_kinds}
    t_sel = {k: 0.0 for k in sched_kinds}
    for c in cases:
        n = math.prod(c["size"])
        gen.manual_seed(c["seed"])
        A = torch.rand(n, dtype=tmap[c["dtype"]], device=dev, generator=gen).mul_(2).sub_(1)
        gen.manual_seed(c["seed"] + 1)
        B = torch.rand(n, dtype=tmap[c["dtype"]], device=dev, generator=gen).mul_(2).sub_(1)
        for k in sched_kinds:
            t0 = time.perf_counter()
            tunings[k].append(choose(k, c))
            t_sel[k] += time.perf_counter() - t0
        plan = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning=tunings[args.schedule][-1])
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
    descs = [p.describe() for _, p, _, _ in items]
    kinds = [kernel_name(d) for d in descs]
    # a staged tile plan with ragged tiles also launches its edge plans (or the ragged-tile kernel)
    launches_per_step = sum(p.launches() for _, p, _, _ in items)
    per_kind = {}
    per_case = []
    for k, (c, plan, A, B) in enumerate(items):
        ms = [evs[s][k][0].elapsed_time(evs[s][k][1]) for s in range(args.steps)]
        d = per_kind.setdefault(kinds[k], [0.0, 0, 0])
        d[0] += sum(ms)
        d[1] += plan.bytes * args.steps
        d[2] += args.steps
        per_case.append(round(plan.bytes / (statistics.median(ms) / 1e3) / 1e9, 1))
    dom = max(per_kind, key=lambda k: per_kind[k][0])
    dom_ms, dom_bytes, dom_n = per_kind[dom]
    peak, peak_src = measured_peak_gbs()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    tr = ncu_traffic_per_gb(dom)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_source": peak_src,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "kernel": dom,
                "launches": dom_n, "algorithmic_bytes_per_launch": int(dom_bytes / dom_n),
                "traffic": (int(tr * dom_bytes / dom_n) if tr else None),
                "split": {k: {"ms": round(v[0], 3), "GBps": round(v[1] / (v[0] / 1e3) / 1e9, 1), "launches": v[2]}
                          for k, v in per_kind.items()},
                "per_case_GBps": per_case, "cases_below_0.7_of_peak": int(sum(g < 0.7 * peak for g in per_case))}

    # the other kinds of schedule on the same resident inputs, timed the same way (back to back)
    schedule_kinds = {args.schedule: {"GBps": round(value, 1), "ms_per_step": round(ms_per_step, 4),
                                      "tuning_seconds": round(t_sel[args.schedule], 1)}}
    for k in sched_kinds[1:]:
        alt = [(c, Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning=tu), A, B)
               for (c, _, A, B), tu in zip(items, tunings[k])]
        ms_k = sweep_pass_ms(alt, args.steps, args.warmup, stream, dev, world)
        schedule_kinds[k] = {"GBps": round(job_throughput(bytes_per_step, world, ms_k), 1),
                             "ms_per_step": round(ms_k, 4), "tuning_seconds": round(t_sel[k], 1)}
        for _, p, _, _ in alt:
            p.close()
    for k in sched_kinds:
        if k != "default":
            schedule_kinds[k]["cases_off_default"] = sum(1 for tu in tunings[k] if tu)
            schedule_kinds[k]["knobs"] = knob_counts(tunings[k])
            schedule_kinds[k]["per_case"] = [plain_json(tu or {}) for tu in tunings[k]]

    # end to end through the public call with pinned host buffers, over the same cases
    pcie = measure_pcie(dev) if rank == 0 or world > 1 else None
    e2e, host = run_e2e(args, items, stream, dev, world, pcie)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_on(items, host, os.cpu_count() or 1, args.cpu_seconds)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GB/s", "cores": os.cpu_count() or 1, "kind": "port",
                   "sample": f"failed: {ex}"}
    del host
    for _, p, _, _ in items:
        p.close()
    items.clear()
    torch.cuda.empty_cache()

    extras = {}
    if world == 1 and not args.no_extras:
        for name, fn in (("reference_gpu", lambda: reference_gpu_summary(args)),
                         ("configs", lambda: configs_summary(args)), ("batched", lambda: batched_summary(args)),
                         ("selector", lambda: selector_summary(args))):
            try:
                extras[name] = fn()
            except Exception as ex:  # an extra never hides the headline
                extras[name] = {"error": f"{type(ex).__name__}: {ex}"}
            torch.cuda.empty_cache()

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded uniform[-1,1])",
                "pct_of_hbm_peak": round(100 * value / world / peak, 2),
                "config": sweep_config(len(cases), bytes_per_step, world),
                "schedules": schedule_note or SCHEDULE_NOTES[args.schedule],
                "schedule_seconds": round(t_sel[args.schedule], 1),
                "schedule_kinds": schedule_kinds,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
                "gpu_launches": launches_per_step * args.steps, **extras}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


SCHEDULE_NOTES = {
    "search": ("measured search per case (TTC's method): every candidate schedule (tile shape x raster x ring "
               "depth and CTAs per SM x tile order x copy form; up to 200) timed, best of 3, and checked bit for "
               "bit against the first; the fastest kept. Chosen before the timed region"),
    "learned": ("learned selector (top-1 on a large predicted gain over the planner default; its top candidates "
                "timed against it on a moderate one). Chosen before the timed region"),
    "default": "planner default",
}


def plain_json(x):
    """`x` with numpy scalars turned into Python numbers, so that json.dumps takes it."""
    return json.loads(json.dumps(x, default=lambda o: o.item() if hasattr(o, "item") else str(o)))


def knob_counts(tunings) -> dict:
    """How many of the cases' schedules set each ttcb_tuning field, with the values that matter for
    the copy form and the tile order (bulk A copies, shifted runs, claimed or round-robin tiles)."""
    out = {}
    for tu in tunings:
        for key, val in (tu or {}).items():
            name = f"{key}={val}" if key in ("bulk_copies", "shifted_runs", "round_robin", "lane_map") else key
            out[name] = out.get(name, 0) + 1
    return dict(sorted(out.items()))


def sweep_pass_ms(items, steps, warmup, stream, dev, world):
    """ms per pass over `items` [(case, plan, A, B)], back to back with CUDA events after `warmup`
    untimed passes; the maximum over ranks."""
    import torch
    import torch.distributed as dist

    def one():
        for c, plan, A, B in items:
            plan(A, B, c["alpha"], c["beta"], stream)
    for _ in range(warmup):
        one()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        one()
    e1.record(stream)
    torch.cuda.synchronize()
    return max_over_ranks(e0.elapsed_time(e1), dev) / steps


# ------------------------------------------------------------------------------------------------
def flushed_timing(plan, A, B, alpha, beta, steps, warmup, flush):
    """Median and best ms of `steps` launches, each after an L2 flush (autotune.L2Flush: 2x the L2
    written, then 2x read; CUDA events)."""
    import torch
    for _ in range(warmup):
        plan(A, B, alpha, beta)
    ms = []
    for _ in range(steps):
        flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        plan(A, B, alpha, beta)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.median(ms), min(ms)


def configs_summary(args, steps=None, warmup=None):
    """The single-problem configurations: TTC's README shape (perm 1,0,2 / 1000,768,16, fp32,
    alpha = beta = 1) and the strided mixed-precision shape (perm 3,1,0,2 / 96,80,72,64, lda + 8,0,4,0;
    z->c with alpha = (0.5, 0.25) and d->s with alpha = 0.5, beta = 0). Inputs uniform[-1,1] from the
    seed (B from seed + 1), resident; the L2 is flushed (2x its size written, then 2x read) before every timed
    launch; CUDA events. Returns {name: result}."""
    import torch
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan
    steps = steps or max(args.steps, 10)
    warmup = warmup or max(args.warmup, 3)
    tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
    from ttc_b200.autotune import L2Flush
    flush = L2Flush()
    peak, _ = measured_peak_gbs()
    out = {}
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
        med, best = flushed_timing(plan, A, B, c["alpha"], c["beta"], steps, warmup, flush)
        d = plan.describe()
        gbs = plan.bytes / (med / 1e3) / 1e9
        out[name] = {"perm": c["perm"], "size": c["size"], "lda": c.get("lda"), "dtype": c["dtype"],
                     "alpha": str(c["alpha"]), "beta": c["beta"], "bytes": plan.bytes,
                     "GBps_median": round(gbs, 1), "GBps_best": round(plan.bytes / (best / 1e3) / 1e9, 1),
                     "frac_of_hbm_peak": round(gbs / peak, 4), "kernel": kernel_name(d), "tile": d.get("tile"),
                     "vec": [d["vecA"], d["vecB"]], "l2": "flushed before every launch (2x L2 written, then 2x read)",
                     "steps": steps,
                     "schedule": "planner default"}
        plan.close()
        # the learned selector's schedule for the same problem (as the sweep uses it)
        try:
            from ttc_b200 import cost_model
            from ttc_b200.autotune import Problem
            tu = cost_model.choose_tuning(Problem(c["perm"], c["size"], c["dtype"], c["alpha"], c["beta"],
                                                  c.get("lda")))
        except Exception as ex:
            tu, out[name]["learned"] = None, {"unavailable": f"{type(ex).__name__}: {ex}"}
        if tu:
            lp = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, lda=c.get("lda"), tuning=tu)
            lmed, lbest = flushed_timing(lp, A, B, c["alpha"], c["beta"], steps, warmup, flush)
            lg = lp.bytes / (lmed / 1e3) / 1e9
            out[name]["learned"] = {"tuning": tu, "GBps_median": round(lg, 1), "frac_of_hbm_peak": round(lg / peak, 4)}
            lp.close()
        elif "learned" not in out[name]:
            out[name]["learned"] = {"tuning": {}, "note": "the selector kept the planner default"}
        # the measured search's winner (TTC's method, as the sweep's `value` uses it)
        try:
            from ttc_b200.autotune import Problem, search
            t0 = time.perf_counter()
            r = search(Problem(c["perm"], c["size"], c["dtype"], c["alpha"], c["beta"], c.get("lda")),
                       max_impl=args.search_candidates, reps=3, verify=True, seed=args.seed)
            secs = time.perf_counter() - t0
            stu = plain_json(dict(r["best"].tuning))
            sp = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, lda=c.get("lda"), tuning=stu or None)
            smed, sbest = flushed_timing(sp, A, B, c["alpha"], c["beta"], steps, warmup, flush)
            sg = sp.bytes / (smed / 1e3) / 1e9
            out[name]["search"] = {"tuning": stu, "candidates": r["candidates"], "tuning_seconds": round(secs, 2),
                                   "GBps_median": round(sg, 1), "frac_of_hbm_peak": round(sg / peak, 4)}
            sp.close()
        except Exception as ex:  # reported, never required
            out[name]["search"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
        torch.cuda.empty_cache()
    return out


def batched_summary(args):
    """The batched workload (4096 problems) in one persistent launch replayed from a CUDA graph,
    against the same problems as a CUDA graph of per-call launches; every batched result compared bit
    for bit with the per-call result. Returns a dict."""
    import torch
    from ttc_b200.batched import Batch
    plans, As, Bs, Cs, t_tune, cases = build_batch_problems(args, 0, torch.device("cuda"))
    batch = Batch(plans, As, Bs, alpha=1.0)
    stream = torch.cuda.current_stream()
    total = batch.bytes
    g = capture_per_call(plans, As, Cs, stream)
    for _ in range(3):
        batch.launch(stream, graph=True)
        g.replay()
    batch.check_status(stream)
    torch.cuda.synchronize()

    def timed(fn, steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_b = timed(lambda: batch.launch(stream, graph=True), 10)
    ms_c = timed(g.replay, 10)
    batch.check_status(stream)
    torch.cuda.synchronize()
    mismatches = sum(0 if torch.equal(b.view(torch.int32), cbuf.view(torch.int32)) else 1 for b, cbuf in zip(Bs, Cs))
    gbs = lambda ms: round(total / (ms / 1e3) / 1e9, 1)
    del g
    batch.close()
    for p in plans:
        p.close()
    return {"workload": BATCH_WORKLOAD, "problems": len(cases), "bytes": total,
            "batched_graph_GBps": gbs(ms_b), "graph_of_per_call_launches_GBps": gbs(ms_c),
            "speedup_vs_graph_of_calls": round(ms_c / ms_b, 2), "schedules": args.batch_tuning,
            "plan_seconds": round(t_tune, 1),
            "mismatches_vs_per_call": mismatches, "steps": 10}


def reference_gpu_summary(args):
    """TTC's own CUDA kernels on this GPU (oracle/_ref/libttc_ref_cuda.so: the first variants of TTC's
    CUDA generator's own order per case, compiled for sm_100a) over the 64-case sweep, on the same
    seeded inputs: per case every built variant is called through TTC's generated wrapper (per-call
    cudaMalloc/cudaMemcpy of the sizes, launch, cudaDeviceSynchronize, cudaFree; CUDAtranspose.py:
    395-429 in the TTC project) and the fastest kept, as TTC's search would. Kernel-only time is the
    device time of TTC's kernels from CUDA's activity records (torch.profiler, min of 3 calls);
    wrapper time is the host wall time of the synchronous call."""
    import torch
    import ttc_b200.workloads as wl
    from oracle import cuda_ref
    from torch.profiler import ProfilerActivity, profile
    ref = cuda_ref.available()
    if ref is None:
        return {"unavailable": "TTC's CUDA kernels were not built (oracle/make_ref_gpu.py needs the TTC sources)"}
    tmap = {"s": torch.float32, "d": torch.float64}
    cases = [c for c in wl.sweep_cases(args.seed)[: args.cases] if ref.covers(c)]
    tot_bytes, t_kernel, t_wrap, chosen = 0, 0.0, 0.0, []
    gen = torch.Generator(device="cuda")
    for c in cases:
        n = math.prod(c["size"])
        gen.manual_seed(c["seed"])
        A = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen).mul_(2).sub_(1)
        gen.manual_seed(c["seed"] + 1)
        B = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen).mul_(2).sub_(1)
        variants = ref.variants(c)
        for j in range(len(variants)):  # warm every variant's module and launch path
            ref.call(c, j, A.data_ptr(), B.data_ptr())
        walls = []
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            for j in range(len(variants)):
                w = float("inf")
                for _ in range(3):
                    t0 = time.perf_counter()
                    ref.call(c, j, A.data_ptr(), B.data_ptr())
                    w = min(w, time.perf_counter() - t0)
                walls.append(w)
        kern = [float("inf")] * len(variants)
        for ev in prof.events():
            if ev.device_type != torch.autograd.DeviceType.CUDA:
                continue
            for j, v in enumerate(variants):
                if v["kernel"] in ev.name:
                    kern[j] = min(kern[j], ev.device_time_total * 1e-6)
        best = min(range(len(variants)), key=lambda j: kern[j])
        tot_bytes += wl.case_bytes(c)
        t_kernel += kern[best]
        t_wrap += walls[best]
        chosen.append(variants[best]["version"])
        del A, B
    torch.cuda.empty_cache()
    m = ref.manifest
    return {"cases": len(cases), "variants_per_case": m["variants_per_case"],
            "kernel_GBps": round(tot_bytes / t_kernel / 1e9, 1), "wrapper_GBps": round(tot_bytes / t_wrap / 1e9, 1),
            "chosen_versions": chosen, "nvcc": " ".join(m["nvcc_flags"]),
            "note": ("TTC's CUDA generator (--maxImplementations 200 ordering), first variants per case compiled "
                     "for sm_100a; fastest by kernel device time on this GPU")}


def selector_summary(args):
    """The learned selector against a fresh measured search on held-out problems (the first
    `--selector-cases` problems of the held-out seed, 1-256 MiB): see cost_model.fresh_head_to_head."""
    import ttc_b200.workloads as wl
    from ttc_b200 import cost_model
    out = cost_model.fresh_head_to_head(wl.learning_cases(cost_model.HELDOUT_SEED, args.selector_cases))
    out["held_out_seed"] = cost_model.HELDOUT_SEED
    return out


# ------------------------------------------------------------------------------------------------
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
    plan = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0, tuning=json.loads(args.tuning) if args.tuning else None)
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


def run_batchcase(args):
    """The batched workload with the planner's schedules (no per-problem search), one persistent
    launch `--reps` times; prints the mean GB/s (CUDA events). Meant to sit under a profiler."""
    import torch
    from ttc_b200.batched import Batch
    args.batch_tuning = "default"
    plans, As, Bs, Cs, _, cases = build_batch_problems(args, 0, torch.device("cuda"))
    batch = Batch(plans, As, Bs, alpha=1.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.reps):
        batch.launch()
    e1.record()
    torch.cuda.synchronize()
    batch.check_status()
    ms = e0.elapsed_time(e1) / max(args.reps, 1)
    print(json.dumps({"workload": "batchcase", "problems": len(cases), "bytes": batch.bytes,
                      "GBps": round(batch.bytes / (ms / 1e3) / 1e9, 1)}), flush=True)
    batch.close()
    for p in plans:
        p.close()
    return 0


def run_configs(args):
    out = configs_summary(args)
    print(json.dumps({"workload": "configs", "steps": max(args.steps, 10), "warmup": max(args.warmup, 3),
                      "l2": "flushed", "results": list(out.values())}), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
BATCH_WORKLOAD = ("batched4096: seeded rank-3..5 fp32 transpositions, random perms, element counts "
                  "log-normal median 64Ki clipped to [1Ki, 1Mi], alpha=1 beta=0")


def build_batch_problems(args, rank, dev):
    """Plans (with per-problem schedules from the measured search), seeded A, and NaN-filled B and C
    buffers of the batched workload. Returns (plans, As, Bs, Cs, tuning seconds, cases)."""
    import torch
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan
    from ttc_b200.autotune import Problem, tune_for_batch
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
    return plans, As, Bs, Cs, time.perf_counter() - t_tune, cases


def capture_per_call(plans, As, Cs, stream):
    """A CUDA graph of every problem's own per-call launch (into Cs)."""
    import torch
    g = torch.cuda.CUDAGraph()
    s2 = torch.cuda.Stream()
    s2.wait_stream(stream)
    with torch.cuda.stream(s2):
        for p, a, cbuf in zip(plans, As, Cs):  # warm the plans' launch paths before capture
            p(a, cbuf, 1.0, 0.0, s2)
        with torch.cuda.graph(g, stream=s2):
            for p, a, cbuf in zip(plans, As, Cs):
                p(a, cbuf, 1.0, 0.0, s2)
    stream.wait_stream(s2)
    return g


def run_batched(args, rank, world, local):
    """Batched mode: every problem of the batch in one persistent launch (plain and replayed from a
    captured CUDA graph) against the same problems launched one call at a time: a Python loop over
    the public call, that loop captured into a CUDA graph, and a loop that synchronizes after every
    call as TTC's generated wrapper does. Every batched result is compared bit for bit with the
    per-call result."""
    import torch
    import torch.distributed as dist
    from ttc_b200.batched import Batch

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    plans, As, Bs, Cs, t_tune, cases = build_batch_problems(args, rank, dev)
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
    g = capture_per_call(plans, As, Cs, stream)
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
    if args.workload == "batchcase":
        return run_batchcase(args)
    return run_sweep(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
