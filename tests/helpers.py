"""Shared helpers for the tests: seeded inputs, bit-exact comparison, TTC's case matrix."""
from __future__ import annotations

import numpy as np

NP = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}
UINT = {"s": np.uint32, "d": np.uint64, "c": np.uint64, "z": np.uint64}


def split(dtype):
    return (dtype[0], dtype[1]) if len(dtype) == 2 else (dtype, dtype)


def buffer_len(size, perm, lda=None, ldb=None):
    la = list(lda) if lda else list(size)
    lb = list(ldb) if ldb else [size[p] for p in perm]
    na = int(np.prod(la[:-1], dtype=np.int64)) * int(size[-1])
    nb = int(np.prod(lb[:-1], dtype=np.int64)) * int(size[perm[-1]])
    return max(na, 1), max(nb, 1)


def uniform(n, letter, seed):
    """uniform[-1, 1] from numpy's default_rng(seed); complex: independent re and im."""
    rng = np.random.default_rng(seed)
    if letter in ("c", "z"):
        real = np.float32 if letter == "c" else np.float64
        re = rng.uniform(-1.0, 1.0, n).astype(real)
        im = rng.uniform(-1.0, 1.0, n).astype(real)
        out = np.empty(n, NP[letter])
        out.real = re
        out.imag = im
        return out
    return rng.uniform(-1.0, 1.0, n).astype(NP[letter])


def make_inputs(size, perm, dtype, seed, lda=None, ldb=None):
    ta, tb = split(dtype)
    na, nb = buffer_len(size, perm, lda, ldb)
    return uniform(na, ta, seed), uniform(nb, tb, seed + 1)


def bits(x: np.ndarray) -> np.ndarray:
    """Raw bit patterns (complex -> pairs), for bit-exact comparison including -0.0 and NaN payloads."""
    if x.dtype == np.complex64:
        return x.view(np.uint32)
    if x.dtype == np.complex128:
        return x.view(np.uint64)
    return x.view(np.uint32 if x.dtype == np.float32 else np.uint64)


def assert_bitexact(got: np.ndarray, want: np.ndarray, what=""):
    """Bit-for-bit equality, except that NaN payloads are not compared (the GPU returns its
    canonical NaN where the host propagates an operand's payload; IEEE 754 leaves this open)."""
    gb, wb = bits(got).copy(), bits(want).copy()
    real = np.float32 if gb.dtype == np.uint32 else np.float64
    gn, wn = np.isnan(gb.view(real)), np.isnan(wb.view(real))
    if not np.array_equal(gn, wn):
        i = int(np.nonzero(gn != wn)[0][0])
        raise AssertionError(f"{what}: NaN positions differ, first at word {i}")
    gb[gn] = 0
    wb[wn] = 0
    if not np.array_equal(gb, wb):
        bad = np.nonzero(gb != wb)[0]
        i = int(bad[0])
        raise AssertionError(f"{what}: {len(bad)} of {gb.size} words differ; first at word {i}: "
                             f"got {got.reshape(-1).view(gb.dtype)[i]:#x} want {want.reshape(-1).view(wb.dtype)[i]:#x}")


def ulp_diff(got: np.ndarray, want: np.ndarray) -> int:
    """Max distance in units in the last place over real components (signed-magnitude ordering)."""
    def ordered(x):
        b = bits(x).astype(np.int64)
        width = 32 if bits(x).dtype == np.uint32 else 64
        sign = np.int64(1) << np.int64(width - 1)
        if width == 64:
            b = bits(x).view(np.int64)
            return np.where(b < 0, np.iinfo(np.int64).min - b, b)
        return np.where(b & sign, -(b & (sign - 1)), b)
    return int(np.max(np.abs(ordered(got) - ordered(want)))) if got.size else 0


# TTC's own test matrix (test-framework/ttc_test.py:80-92)
TTC_DTYPES = ["d", "s", "c", "z", "sd", "ds", "cz", "zc"]
TTC_ALPHA = [1.1]
TTC_BETAS = [1, -1, 1.2, 0]
TTC_PERMS = [[2, 0, 1], [1, 0], [0, 2, 1], [1, 2, 0], [1, 0, 2], [2, 1, 0], [3, 1, 0, 2]]
TTC_SIZES = [
    [[11, 8, 3], [16, 4, 25]],
    [[7, 3], [7, 8], [8, 7], [8, 8], [16, 11], [11, 16], [17, 17], [17, 23]],
    [[11, 8, 3], [1, 4, 3], [11, 7, 17], [11, 17, 7], [7, 32, 32]],
    [[11, 8, 3], [4, 4, 3], [12, 8, 17], [33, 17, 7], [32, 32, 4]],
    [[11, 8, 3], [16, 16, 3], [12, 8, 17], [33, 17, 7], [32, 32, 4]],
    [[11, 8, 3], [16, 4, 25], [12, 8, 17], [33, 17, 9], [32, 32, 4]],
    [[17, 3, 7, 9]],
]


def ttc_cases():
    """The reference sweep: alpha/beta x dtype over the first two perms, then every perm and size
    with beta = 0 and with beta = 1.1 (ttc_test.py:174-217)."""
    cases = []
    for beta in TTC_BETAS:
        for dt in TTC_DTYPES:
            for c in range(2):
                for size in TTC_SIZES[c]:
                    cases.append((TTC_PERMS[c], size, dt, 1.1, beta))
    for beta, alpha in ((0.0, 1.1), (1.1, 1.0)):
        for c in range(len(TTC_SIZES)):
            for dt in TTC_DTYPES:
                for size in TTC_SIZES[c]:
                    cases.append((TTC_PERMS[c], size, dt, alpha, beta))
    return cases
