"""The allocation-free entry point ttcb_transpose_noalloc(), called through the C ABI.

It serves callers that may not allocate device memory where they transpose (memory owned by an
external pool, or a section where cudaMalloc is forbidden): its descriptor lives in a fixed scratch
array inside the library instead of a cudaMalloc'd buffer. Its results must equal the oracle's and
the plan-based entry point's bit for bit, on two calls in a row (the second reuses the scratch the
first wrote). A plan made before a no-allocation call must still launch afterwards (the entry point
never lowers a kernel's shared-memory limit), and a call on a stream under capture is refused.
This file is named to be collected last, so a run that stops at the first failure has run every
other test before it; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

CASES = [
    ([1, 0, 2], [300, 257, 5], "s", 1.0, 0.5, None, None),
    ([2, 0, 3, 1], [13, 9, 6, 11], "d", -1.5, 0.0, [16, 10, 6, 12], [6, 15, 12, 9]),
    ([3, 1, 0, 2], [24, 20, 18, 16], "zc", complex(0.5, 0.25), 0.0, [26, 20, 19, 16], None),
    ([0, 2, 1], [40, 33, 17], "c", complex(1.0, -2.0), complex(0.5, 0.5), None, None),
    ([1, 0], [7, 20001], "s", 2.0, 0.0, None, None),
]


def _noalloc(A, B, perm, size, lda, ldb, dtype, alpha, beta, stream=None):
    """Calls the entry point; returns its status (0 = TTCB_OK)."""
    import torch
    from ttc_b200 import _native
    from ttc_b200.core import pack_scalar, split_dtype
    from ttc_b200._native import i32, i64
    ta, tb = split_dtype(dtype)
    al = pack_scalar(ta, alpha)
    be = pack_scalar(tb, beta) if complex(beta) != 0 else None
    st = stream if stream is not None else torch.cuda.current_stream()
    return _native.lib().ttcb_transpose_noalloc(
        len(size), i32(perm), i64(size), i64(lda) if lda else None, i64(ldb) if ldb else None,
        _native.DTYPES[ta], _native.DTYPES[tb], A.data_ptr(), B.data_ptr(), ctypes.cast(al, ctypes.c_void_p),
        ctypes.cast(be, ctypes.c_void_p) if be is not None else None, st.cuda_stream)


@pytest.mark.parametrize("case", CASES, ids=[f"{c[2]}-{c[0]}" for c in CASES])
def test_noalloc_matches_oracle_and_plan_entry_point_twice(case):
    import torch
    from ttc_b200 import Plan
    from ttc_b200._native import check
    from helpers import assert_bitexact, make_inputs
    perm, size, dtype, alpha, beta, lda, ldb = case
    for call in range(2):
        A, B = make_inputs(size, perm, dtype, 40 + call, lda, ldb)
        want = oracle.transpose(A, B.copy(), perm, size, alpha, beta, lda, ldb, dtype)
        dA = torch.from_numpy(A).cuda()
        ref = torch.from_numpy(B).cuda()
        got = ref.clone()
        plan = Plan(perm, size, dtype, complex(beta) != 0, lda, ldb)
        plan(dA, ref, alpha, beta)
        check(_noalloc(dA, got, perm, size, lda, ldb, dtype, alpha, beta))
        torch.cuda.synchronize()
        assert_bitexact(got.cpu().numpy(), want, f"no-allocation call {call} vs oracle {case}")
        assert_bitexact(got.cpu().numpy(), ref.cpu().numpy(), f"no-allocation call {call} vs plan {case}")
        plan.close()


def test_plan_made_before_a_noalloc_call_still_launches():
    """A plan whose staged kernel needs more shared memory than a later no-allocation call of the
    same kernel instantiation: the no-allocation call must not lower the kernel's limit."""
    import torch
    from ttc_b200 import Plan
    from ttc_b200.core import plan_host_json
    from ttc_b200._native import check
    from helpers import assert_bitexact, make_inputs
    big, small = [1024, 1024], [2048, 1024]
    pb = plan_host_json([1, 0], big, "d", False)
    ps = plan_host_json([1, 0], small, "d", False, tuning={"kernel": 1})
    # same instantiation (fp64, 16-byte accesses, register path, streaming stores), larger staging
    assert (pb["vecA"], pb["vecB"], pb["tile"]["reg"]) == (ps["vecA"], ps["vecB"], ps["tile"]["reg"])
    assert pb["tile"]["smem_async"] > ps["tile"]["smem_async"] > 48 * 1024 - 2048
    plan = Plan([1, 0], big, "d", False)
    A2, B2 = make_inputs(small, [1, 0], "d", 5)
    dA2, dB2 = torch.from_numpy(A2).cuda(), torch.from_numpy(B2).cuda()
    check(_noalloc(dA2, dB2, [1, 0], small, None, None, "d", 1.0, 0.0))
    A, B = make_inputs(big, [1, 0], "d", 6)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    plan(dA, dB, 1.0, 0.0)
    torch.cuda.synchronize()
    assert_bitexact(dB.cpu().numpy(), oracle.transpose(A, B.copy(), [1, 0], big, 1.0, 0.0, dtype="d"), "plan after")
    assert_bitexact(dB2.cpu().numpy(), oracle.transpose(A2, B2.copy(), [1, 0], small, 1.0, 0.0, dtype="d"),
                    "no-allocation call")
    plan.close()


def test_noalloc_refuses_a_stream_under_capture():
    """The descriptor upload reads host memory that lives only during the call; under capture the
    call returns TTCB_ERR_UNSUPPORTED and enqueues nothing (the captured graph stays empty)."""
    import torch
    from ttc_b200 import _native
    perm, size = [1, 0], [64, 48]
    dA = torch.zeros(64 * 48, device="cuda")
    dB = torch.zeros(64 * 48, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            st = _noalloc(dA, dB, perm, size, None, None, "s", 1.0, 0.0, stream=s)
        finally:
            g.capture_end()
    assert st == 9, _native.last_error()  # TTCB_ERR_UNSUPPORTED
    assert "captured" in _native.last_error()
    del g
    torch.cuda.synchronize()
