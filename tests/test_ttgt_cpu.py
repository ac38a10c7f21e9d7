"""Tensor contractions through transpositions (ttc_b200.ttgt), host side: the mode classes and the
three permutations that plan_contraction gives, replayed with numpy on column-major buffers (the
transposition as np.transpose, the GEMM as a batched matrix product laid out as the GPU path lays it
out), must reproduce numpy.einsum."""
import math

import numpy as np
import pytest

from ttc_b200 import TTCError
from ttc_b200.ttgt import plan_contraction

PATTERNS = [("ab", "bc", "ac"), ("abc", "cbd", "ad"), ("abcd", "dbe", "eca"), ("ijk", "jl", "lki"),
            ("mab", "mbc", "mac"), ("xay", "ybx", "axb"), ("ab", "cd", "acbd"), ("abc", "bc", "a"),
            ("pqrs", "srt", "ptq")]


def _replay(a, b, c, ext, A, B, alpha, beta, C):
    p = plan_contraction(a, b, c)
    nd = lambda flat, s: flat.reshape([ext[m] for m in s], order="F")
    Am = np.transpose(nd(A, a), p["perm_a"]).reshape(-1, order="F")
    Bm = np.transpose(nd(B, b), p["perm_b"]).reshape(-1, order="F")
    n = lambda s: math.prod(ext[m] for m in s)
    M, K, N, L = n(p["free_a"]), n(p["contracted"]), n(p["free_b"]), n(p["batch"])
    Ct = np.matmul(Bm.reshape(L, N, K), Am.reshape(L, K, M)).reshape(-1)
    Cn = np.transpose(nd(Ct, p["c_mat"]), p["perm_c"]).reshape(-1, order="F")
    return alpha * Cn + beta * C


@pytest.mark.parametrize("a,b,c", PATTERNS)
def test_plan_replays_to_einsum(a, b, c):
    rng = np.random.default_rng(len(a + b + c))
    ext = {m: int(rng.integers(2, 6)) for m in set(a + b + c)}
    A = rng.standard_normal(math.prod(ext[m] for m in a))
    B = rng.standard_normal(math.prod(ext[m] for m in b))
    C = rng.standard_normal(math.prod(ext[m] for m in c))
    got = _replay(a, b, c, ext, A, B, 0.5, -1.5, C)
    nd = lambda flat, s: flat.reshape([ext[m] for m in s], order="F")
    want = 0.5 * np.einsum(f"{a},{b}->{c}", nd(A, a), nd(B, b)).reshape(-1, order="F") - 1.5 * C
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)


def test_mode_classes():
    p = plan_contraction("mabk", "mbck", "mack")
    assert (p["free_a"], p["free_b"], p["contracted"], p["batch"]) == ("a", "c", "b", "mk")
    p = plan_contraction("ab", "bc", "ac")
    assert p["perm_a"] == [0, 1] and p["perm_b"] == [0, 1] and p["perm_c"] == [0, 1]


def test_invalid_modes_are_rejected():
    with pytest.raises(TTCError):
        plan_contraction("aab", "bc", "ac")  # repeated mode
    with pytest.raises(TTCError):
        plan_contraction("abz", "bc", "ac")  # z in A only
    with pytest.raises(TTCError):
        plan_contraction("ab", "bc", "acy")  # y in C only
