"""Host-side checks of the allocation-free entry point (no GPU needed).

Its problems are planned on the host before any CUDA call, so the rejection of a descriptor larger
than the scratch array is reachable on the CPU; the test lowers the accepted size through a test
hook so that an ordinary problem reaches it. A second check confirms that the descriptors the
planner produces with its default tile limits stay well inside the 64 KiB scratch array.
"""
import ctypes

from ttc_b200 import _native
from ttc_b200._native import i32, i64


def _call(perm, size, dtype="s"):
    al = (ctypes.c_float * 1)(1.0)
    fake_a, fake_b = 0x10000, 0x20000  # never dereferenced: these calls return before any CUDA work
    return _native.lib().ttcb_transpose_noalloc(len(size), i32(perm), i64(size), None, None, _native.DTYPES[dtype],
                                                _native.DTYPES[dtype], fake_a, fake_b,
                                                ctypes.cast(al, ctypes.c_void_p), None, None)


def test_descriptor_over_the_limit_is_rejected_before_any_cuda_call():
    lib = _native.lib()
    full = lib.ttcb_test_noalloc_limit(1024)
    try:
        assert full == 64 * 1024
        st = _call([1, 0, 2], [300, 257, 5])
        assert st == 9, _native.last_error()  # TTCB_ERR_UNSUPPORTED
        msg = _native.last_error()
        assert "bytes of scratch" in msg and "at most 1024" in msg, msg
    finally:
        lib.ttcb_test_noalloc_limit(0)


def test_bad_arguments_are_rejected_before_any_cuda_call():
    assert _call([0, 0], [4, 4]) == 3  # TTCB_ERR_BAD_PERM
    assert _call([1, 0], [4, -1]) == 1  # TTCB_ERR_INVALID_ARG (negative extent)


def test_largest_default_descriptors_fit_the_scratch_array():
    """Descriptor bytes = header + 8 per A and B run segment + 4 per tile element; the planner caps a
    default tile at 16 KiB of A elements and 1024 segments a side, so no default plan comes near
    64 KiB. Checked on the tiles the planner picks for a few extreme shapes."""
    layout = (ctypes.c_int64 * 13)()
    _native.lib().ttcb_test_desc_layout(layout)
    header = layout[0]
    worst = 0
    for perm, size, dt in [([1, 0], [4096, 4096], "s"), ([1, 0], [4096, 4096], "d"), ([2, 1, 0], [4, 1024, 4], "s"),
                           ([1, 0, 3, 2], [4, 4, 256, 256], "s"), ([3, 2, 1, 0], [8, 8, 8, 8192], "z")]:
        n = _native.lib().ttcb_test_plan_host_desc(len(size), i32(perm), i64(size), None, None, _native.DTYPES[dt],
                                                   _native.DTYPES[dt], 0, None, None, None, 0)
        worst = max(worst, n)
    assert header < worst < 48 * 1024
