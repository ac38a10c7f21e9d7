"""Tensor contractions staged through this library's transpositions (TTGT: transpose, transpose,
GEMM, transpose).

    C[c] = alpha * sum over the contracted modes of A[a] * B[b] + beta * C[c]

A transposition is rarely an end in itself. Its commonest caller is a tensor contraction that is
cast as a matrix product, whose operands must first be laid out as matrices. This module does that
with the sm_100a transposition kernels and cuBLAS (through torch.bmm):

1. A is transposed to (free modes of A, contracted modes, batch modes), an M x K matrix per batch;
2. B is transposed to (contracted modes, free modes of B, batch modes), a K x N matrix per batch;
3. one batched GEMM gives the M x N matrices of (free A, free B, batch);
4. a last transposition puts them in C's mode order and applies alpha and beta (the kernels' own
   ``alpha * perm(X) + beta * C``).

A step whose permutation is the identity is skipped (step 4 then still applies alpha and beta).
Tensors are flat CUDA tensors in TTC's column-major layout: the first mode of each mode string
varies fastest. Modes are single characters; a mode in A and B but not C is contracted, in all
three a batch mode, in one operand and C a free mode. A mode in one operand only is not supported.
The steps' intermediates are allocated with torch (this is a convenience layer above the C ABI,
not a path that avoids allocation).
"""
from __future__ import annotations

import math
from typing import Optional

from ._native import TTCError
from .core import Plan, torch_letter

_plans: dict = {}


def plan_contraction(a: str, b: str, c: str) -> dict:
    """Mode classes and the three transpositions of a contraction (host only).

    Returns {"free_a", "free_b", "contracted", "batch"} (mode strings) and the mode orders of the
    A matrix, the B matrix and the GEMM result, with the TTC permutations that produce them
    ("perm_a", "perm_b", "perm_c": perm[j] is the source position of the target's j-th mode)."""
    for name, s in (("A", a), ("B", b), ("C", c)):
        if len(set(s)) != len(s):
            raise TTCError(1, f"repeated mode in {name}'s modes {s!r}")
    only = (set(a) - set(b) - set(c)) | (set(b) - set(a) - set(c)) | (set(c) - set(a) - set(b))
    if only:
        raise TTCError(1, f"modes {sorted(only)} appear in one tensor only")
    batch = "".join(m for m in c if m in a and m in b)
    free_a = "".join(m for m in a if m in c and m not in b)
    free_b = "".join(m for m in b if m in c and m not in a)
    contracted = "".join(m for m in a if m in b and m not in c)
    a_mat = free_a + contracted + batch
    b_mat = contracted + free_b + batch
    c_mat = free_a + free_b + batch
    return {"free_a": free_a, "free_b": free_b, "contracted": contracted, "batch": batch,
            "a_mat": a_mat, "b_mat": b_mat, "c_mat": c_mat,
            "perm_a": [a.index(m) for m in a_mat], "perm_b": [b.index(m) for m in b_mat],
            "perm_c": [c_mat.index(m) for m in c]}


def _transpose(src, dst, perm, size, alpha, beta, stream):
    dtype = torch_letter(src)
    key = (tuple(perm), tuple(size), dtype, complex(beta) != 0, src.device.index)
    plan = _plans.get(key)
    if plan is None:
        plan = _plans[key] = Plan(perm, size, dtype, complex(beta) != 0)
    plan(src, dst, alpha, beta, stream)


def contract(A, a: str, B, b: str, C, c: str, extents: dict, alpha=1.0, beta=0.0, stream=None):
    """``C[c] = alpha * A[a] * B[b] (summed over the contracted modes) + beta * C[c]`` on flat CUDA
    tensors of one dtype (float32, float64, complex64 or complex128), in TTC's column-major layout
    with the extents given per mode. Asynchronous on ``stream`` (default: torch's current stream)."""
    import torch
    p = plan_contraction(a, b, c)
    for name, t, s in (("A", A, a), ("B", B, b), ("C", C, c)):
        missing = [m for m in s if m not in extents]
        if missing:
            raise TTCError(1, f"no extent for modes {missing}")
        if t.numel() != math.prod(extents[m] for m in s):
            raise TTCError(1, f"{name} holds {t.numel()} elements, its modes {s!r} give "
                              f"{math.prod(extents[m] for m in s)}")
    if not (A.dtype == B.dtype == C.dtype):
        raise TTCError(5, "A, B and C must have one dtype")
    ext = lambda s: [extents[m] for m in s]
    n = lambda s: math.prod(ext(s))
    st = stream if stream is not None else torch.cuda.current_stream()
    with torch.cuda.stream(st):
        if p["perm_a"] == list(range(len(a))):
            Am = A
        else:
            Am = torch.empty_like(A)
            _transpose(A, Am, p["perm_a"], ext(a), 1.0, 0.0, st)
        if p["perm_b"] == list(range(len(b))):
            Bm = B
        else:
            Bm = torch.empty_like(B)
            _transpose(B, Bm, p["perm_b"], ext(b), 1.0, 0.0, st)
        M, K, N, L = n(p["free_a"]), n(p["contracted"]), n(p["free_b"]), n(p["batch"])
        # column-major M x K per batch is row-major K x M: C^T = B^T A^T, row-major N x M per batch
        Cm = torch.bmm(Bm.view(L, N, K), Am.view(L, K, M)).reshape(-1)
        _transpose(Cm, C, p["perm_c"], ext(p["c_mat"]), alpha, beta, st)
    return C
