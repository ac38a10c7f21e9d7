"""Tensor contractions through transpositions (ttc_b200.ttgt) on the GPU: the sm_100a transposition
kernels stage the operands and the result around one cuBLAS batched GEMM. Results against numpy's
einsum in float64; the tolerance is the GEMM's (the transpositions themselves are exact):
|got - want| <= tol * (|alpha| * sum_k |A||B| + |beta| |C|), tol = 1e-4 for fp32 / complex64 and
1e-12 for fp64 / complex128."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PATTERNS = [("ab", "bc", "ac"), ("abc", "cbd", "ad"), ("abcd", "dbe", "eca"), ("ijk", "jl", "lki"),
            ("mab", "mbc", "mac"), ("xay", "ybx", "axb"), ("ab", "cd", "acbd"), ("abc", "bc", "a")]


@pytest.mark.parametrize("dtype", ["s", "d", "c", "z"])
@pytest.mark.parametrize("a,b,c", PATTERNS)
def test_contraction_matches_einsum(a, b, c, dtype):
    import torch
    from ttc_b200.ttgt import contract
    tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
    rng = np.random.default_rng(len(a) * 7 + len(b))
    ext = {m: int(rng.integers(3, 40)) for m in set(a + b + c)}
    while math.prod(ext[m] for m in set(a + b + c)) > 4_000_000:
        k = max(ext, key=ext.get)
        ext[k] = max(2, ext[k] // 2)

    def rand(n):
        x = rng.uniform(-1, 1, n)
        return x + 1j * rng.uniform(-1, 1, n) if dtype in "cz" else x

    A, B, C = (rand(math.prod(ext[m] for m in s)) for s in (a, b, c))
    alpha, beta = (complex(0.5, -0.25), complex(-1.5, 0.5)) if dtype in "cz" else (0.5, -1.5)
    nd = lambda flat, s: flat.reshape([ext[m] for m in s], order="F")
    want = alpha * np.einsum(f"{a},{b}->{c}", nd(A, a), nd(B, b)).reshape(-1, order="F") + beta * C
    mag = abs(alpha) * np.einsum(f"{a},{b}->{c}", np.abs(nd(A, a)), np.abs(nd(B, b))).reshape(-1, order="F") \
        + abs(beta) * np.abs(C)
    dA, dB, dC = (torch.from_numpy(x.astype(np.dtype(tmap[dtype].__str__().split(".")[-1]))).cuda() for x in (A, B, C))
    contract(dA, a, dB, b, dC, c, ext, alpha, beta)
    got = dC.cpu().numpy().astype(np.complex128 if dtype in "cz" else np.float64)
    tol = 1e-4 if dtype in "sc" else 1e-12
    assert np.all(np.abs(got - want) <= tol * mag + 1e-30), (a, b, c, dtype, float(np.max(np.abs(got - want) / (mag + 1e-30))))
