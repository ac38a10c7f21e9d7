"""Pins the oracle: it must reproduce, bit for bit, the outputs of TTC's own generated reference loop
(tests/golden/ttc_reference_loop.npz, made by tests/golden/make_golden.py from the TTC sources), and
an independent numpy restatement of the update rules."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, make_inputs, split

GOLDEN = Path(__file__).resolve().parent / "golden" / "ttc_reference_loop.npz"


def load_golden():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]).decode())
    return meta["cases"], z


def _inputs_checked(c):
    import hashlib
    A, B = make_inputs(c["size"], c["perm"], c["dtype"], c["seed"], c["lda"], c["ldb"])
    assert hashlib.sha256(A.tobytes()).hexdigest() == c["sha_A"], "seeded inputs changed (numpy RNG stream?)"
    assert hashlib.sha256(B.tobytes()).hexdigest() == c["sha_B"]
    return A, B


def test_oracle_matches_ttc_generated_reference_loop():
    cases, z = load_golden()
    assert len(cases) >= 250
    for k, c in enumerate(cases):
        A, B = _inputs_checked(c)
        got = oracle.transpose(A, B.copy(), c["perm"], c["size"], c["alpha"], c["beta"], c["lda"], c["ldb"],
                               c["dtype"])
        assert_bitexact(got, z[f"B{k}"], f"golden case {k}: {c}")


def test_oracle_parallel_form_matches_serial():
    cases, z = load_golden()
    for k, c in enumerate(cases[::7]):
        A, B = make_inputs(c["size"], c["perm"], c["dtype"], c["seed"], c["lda"], c["ldb"])
        s = oracle.transpose(A, B.copy(), c["perm"], c["size"], c["alpha"], c["beta"], c["lda"], c["ldb"], c["dtype"])
        p = oracle.transpose(A, B.copy(), c["perm"], c["size"], c["alpha"], c["beta"], c["lda"], c["ldb"], c["dtype"],
                             threads=4)
        assert_bitexact(p, s, f"parallel vs serial {c}")


def _numpy_reference(A, B, perm, size, alpha, beta, dtype):
    """Independent restatement in numpy, one rounding per operation (dense layouts only)."""
    ta, tb = split(dtype)
    nd = len(size)
    Ar = A.reshape(tuple(reversed(size)))  # row-major view of a column-major tensor
    Bp = np.transpose(Ar, [nd - 1 - perm[j] for j in reversed(range(nd))]).reshape(-1)
    if ta in "sd":
        at = np.float32 if ta == "s" else np.float64
        bt = np.float32 if tb == "s" else np.float64
        t = (at(alpha) * Bp).astype(at)
        if beta == 0:
            return t.astype(bt)
        u = (bt(beta) * B).astype(bt)
        return (t.astype(np.float64) + u.astype(np.float64)).astype(bt) if (ta, tb) in (("d", "s"), ("s", "d")) \
            else (t + u).astype(bt)
    rt_a = np.float32 if ta == "c" else np.float64
    rt_b = np.float32 if tb == "c" else np.float64
    ar, ai = rt_a(np.real(alpha)), rt_a(np.imag(alpha))
    xr, xi = Bp.real.astype(rt_a), Bp.imag.astype(rt_a)
    tr = (ar * xr).astype(rt_a) - (ai * xi).astype(rt_a)
    ti = (ar * xi).astype(rt_a) + (ai * xr).astype(rt_a)
    tr, ti = tr.astype(rt_b), ti.astype(rt_b)
    if beta != 0:
        br, bi = rt_b(np.real(beta)), rt_b(np.imag(beta))
        yr, yi = B.real.astype(rt_b), B.imag.astype(rt_b)
        tr = tr + ((br * yr).astype(rt_b) - (bi * yi).astype(rt_b))
        ti = ti + ((br * yi).astype(rt_b) + (bi * yr).astype(rt_b))
    out = np.empty(B.shape, B.dtype)
    out.real, out.imag = tr, ti
    return out


@pytest.mark.parametrize("dtype", ["s", "d", "c", "z", "sd", "cz"])
def test_oracle_matches_numpy_restatement(dtype):
    rng = np.random.default_rng(5)
    for it in range(20):
        r = int(rng.integers(1, 5))
        size = [int(x) for x in rng.integers(1, 9, r)]
        perm = [int(x) for x in rng.permutation(r)]
        A, B = make_inputs(size, perm, dtype, it)
        ta, _ = split(dtype)
        alpha = complex(1.25, -0.5) if ta in "cz" else 1.25
        beta = [0.0, -0.75][it % 2]
        if ta in "cz" and beta:
            beta = complex(beta, 0.5)
        want = _numpy_reference(A, B.copy(), perm, size, alpha, beta, dtype)
        got = oracle.transpose(A, B.copy(), perm, size, alpha, beta, dtype=dtype)
        assert_bitexact(got, want, f"{dtype} {perm} {size}")


def test_oracle_rejects_bad_arguments():
    A = np.zeros(100, np.float32)
    B = np.zeros(100, np.float32)
    with pytest.raises(ValueError):
        oracle.transpose(A, B, [1, 0], [5, 5], ldb=[4, 5])
    with pytest.raises(ValueError):
        oracle.transpose(A, B, [1, 0], [50, 5])
