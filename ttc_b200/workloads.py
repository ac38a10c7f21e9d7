"""Seeded synthetic workloads with the shapes of the reference's benchmark method.

TTC benchmarks 200 MiB rank-2..6 transpositions (README.md:84, benchmark/benchmark.py:39-191 in the
TTC project); these generators produce seeded cases of those sizes and value distributions. No
dataset is read: every tensor is filled from a seeded uniform[-1, 1] generator.
"""
from __future__ import annotations

import math

import numpy as np

MIB = 1 << 20
ELEM = {"s": 4, "d": 8, "c": 8, "z": 16}


def readme_case() -> dict:
    """perm 1,0,2 / size 1000,768,16, fp32 A and B, alpha = beta = 1 (TTC README example)."""
    return {"perm": [1, 0, 2], "size": [1000, 768, 16], "dtype": "s", "alpha": 1.0, "beta": 1.0}


def _extents(rng, d: int, n_target: float, forced_dim: int, forced: int, min_ext: int = 2) -> list[int]:
    """Log-uniform extents with one forced extent, rescaled so the product is ~n_target."""
    w = rng.uniform(0.0, 1.0, d)
    w[forced_dim] = 0.0
    others = [i for i in range(d) if i != forced_dim]
    budget = math.log(n_target / forced)
    if not others:
        return [forced]
    wsum = float(sum(w[i] for i in others)) or 1.0
    size = [0] * d
    size[forced_dim] = forced
    for i in others:
        size[i] = max(min_ext, int(round(math.exp(budget * w[i] / wsum))))
    # rescale the largest free extent so the total matches the target
    big = max(others, key=lambda i: size[i])
    rest = forced * math.prod(size[i] for i in others if i != big)
    size[big] = max(min_ext, int(round(n_target / rest)))
    return size


def sweep_cases(seed: int = 2024, count: int = 64, mib: float = 200.0) -> list[dict]:
    """The large sweep: `count` cases, rank uniform in 2..6, a uniform random non-identity
    permutation, fp32 or fp64, alpha=1/beta=0 for even cases and alpha=1.5/beta=-0.5 for odd
    ones, log-uniform extents with one forced into [7, 31], |A| ~ `mib` MiB."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        d = int(rng.integers(2, 7))
        while True:
            perm = [int(x) for x in rng.permutation(d)]
            if perm != list(range(d)):
                break
        dtype = "s" if rng.random() < 0.5 else "d"
        alpha, beta = (1.0, 0.0) if k % 2 == 0 else (1.5, -0.5)
        n_target = mib * MIB / ELEM[dtype]
        fd = int(rng.integers(0, d))
        forced = int(rng.integers(7, 32))
        size = _extents(rng, d, n_target, fd, forced)
        out.append({"perm": perm, "size": size, "dtype": dtype, "alpha": alpha, "beta": beta, "seed": seed + k})
    return out


def strided_cases() -> list[dict]:
    """Mixed precision with strided sub-tensors: perm 3,1,0,2, extents 96,80,72,64,
    lda = extents + {8,0,4,0}, B dense, beta = 0; z->c with alpha = (0.5, 0.25) and d->s with 0.5."""
    base = {"perm": [3, 1, 0, 2], "size": [96, 80, 72, 64], "lda": [104, 80, 76, 64], "beta": 0.0}
    return [dict(base, dtype="zc", alpha=complex(0.5, 0.25)), dict(base, dtype="ds", alpha=0.5)]


def batched_cases(seed: int = 7, count: int = 4096, median: int = 65536, lo: int = 1024,
                  hi: int = 1 << 20) -> list[dict]:
    """Many small transpositions: rank uniform in {3,4,5}, random permutation, fp32, element counts
    log-normal with the given median clipped to [lo, hi], extents factorised from the count."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        d = int(rng.integers(3, 6))
        perm = [int(x) for x in rng.permutation(d)]
        n = int(np.clip(round(math.exp(rng.normal(math.log(median), 1.0))), lo, hi))
        w = rng.uniform(0.2, 1.0, d)
        logs = math.log(n) * w / w.sum()
        size = [max(1, int(round(math.exp(x)))) for x in logs]
        big = int(np.argmax(size))
        rest = math.prod(s for i, s in enumerate(size) if i != big)
        size[big] = max(1, int(round(n / rest)))
        out.append({"perm": perm, "size": size, "dtype": "s", "alpha": 1.0, "beta": 0.0})
    return out


def learning_cases(seed: int, count: int, mib_lo: float = 1.0, mib_hi: float = 256.0) -> list[dict]:
    """Cases for the learned plan selector: rank 2..6, random permutation, fp32/fp64, |A| log-uniform
    in [mib_lo, mib_hi] MiB, one extent in [7, 31] for half of them, beta != 0 for a third."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        d = int(rng.integers(2, 7))
        perm = [int(x) for x in rng.permutation(d)]
        dtype = "s" if rng.random() < 0.5 else "d"
        mib = math.exp(rng.uniform(math.log(mib_lo), math.log(mib_hi)))
        n_target = mib * MIB / ELEM[dtype]
        fd = int(rng.integers(0, d))
        forced = int(rng.integers(7, 32)) if rng.random() < 0.5 else int(round(n_target ** (1.0 / d)))
        forced = max(2, min(forced, int(n_target)))
        size = _extents(rng, d, n_target, fd, forced)
        beta = -0.5 if rng.random() < 1.0 / 3.0 else 0.0
        out.append({"perm": perm, "size": size, "dtype": dtype, "alpha": 1.0, "beta": beta})
    return out


def case_bytes(c: dict) -> int:
    """Algorithmic bytes: N*(|TA| + |TB|*(1+[beta!=0]))."""
    dt = c["dtype"]
    ta, tb = (dt[0], dt[1]) if len(dt) == 2 else (dt, dt)
    n = math.prod(c["size"])
    return n * (ELEM[ta] + ELEM[tb] * (2 if complex(c["beta"]) != 0 else 1))
