"""The allocation-free entry point ttcb_transpose_noalloc(), called through the C ABI.

It serves callers that may not allocate device memory where they transpose (memory owned by an
external pool, or a section where cudaMalloc is forbidden): its descriptor lives in a fixed scratch
array inside the library instead of a cudaMalloc'd buffer. Its results must equal the plan-based
entry point's bit for bit, on two calls in a row (the second reuses the scratch the first wrote).
This file is named to be collected last, so a run that stops at the first failure has run every
other test before it; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    ([1, 0, 2], [300, 257, 5], "s", 1.0, 0.5, None, None),
    ([2, 0, 3, 1], [13, 9, 6, 11], "d", -1.5, 0.0, [16, 10, 6, 12], [6, 15, 12, 9]),
    ([3, 1, 0, 2], [24, 20, 18, 16], "zc", complex(0.5, 0.25), 0.0, [26, 20, 19, 16], None),
    ([0, 2, 1], [40, 33, 17], "c", complex(1.0, -2.0), complex(0.5, 0.5), None, None),
    ([1, 0], [7, 20001], "s", 2.0, 0.0, None, None),
]


def _noalloc(A, B, perm, size, lda, ldb, dtype, alpha, beta):
    import torch
    from ttc_b200 import _native
    from ttc_b200.core import pack_scalar, split_dtype
    from ttc_b200._native import check, i32, i64
    ta, tb = split_dtype(dtype)
    al = pack_scalar(ta, alpha)
    be = pack_scalar(tb, beta) if complex(beta) != 0 else None
    check(_native.lib().ttcb_transpose_noalloc(
        len(size), i32(perm), i64(size), i64(lda) if lda else None, i64(ldb) if ldb else None,
        _native.DTYPES[ta], _native.DTYPES[tb], A.data_ptr(), B.data_ptr(), ctypes.cast(al, ctypes.c_void_p),
        ctypes.cast(be, ctypes.c_void_p) if be is not None else None, torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("case", CASES, ids=[f"{c[2]}-{c[0]}" for c in CASES])
def test_noalloc_matches_plan_entry_point_twice(case):
    import torch
    from ttc_b200 import Plan
    from helpers import assert_bitexact, make_inputs, split
    perm, size, dtype, alpha, beta, lda, ldb = case
    ta, tb = split(dtype)
    tmap = {"s": torch.float32, "d": torch.float64, "c": torch.complex64, "z": torch.complex128}
    for call in range(2):
        A, B = make_inputs(size, perm, dtype, 40 + call, lda, ldb)
        dA = torch.from_numpy(A).cuda()
        ref = torch.from_numpy(B).cuda()
        got = ref.clone()
        plan = Plan(perm, size, dtype, complex(beta) != 0, lda, ldb)
        plan(dA, ref, alpha, beta)
        _noalloc(dA, got, perm, size, lda, ldb, dtype, alpha, beta)
        torch.cuda.synchronize()
        assert_bitexact(got.cpu().numpy(), ref.cpu().numpy(), f"call {call} {case}")
        plan.close()
