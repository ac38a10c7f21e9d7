"""Python API over the C ABI: plans and the ``transpose(A, B, alpha, beta)`` call.

Tensors are torch CUDA tensors (or raw device pointers); torch supplies device memory and streams
only. All arithmetic happens in the sm_100a kernels of ``libttcb200.so``.
"""
from __future__ import annotations

import ctypes
import json
from typing import Optional, Sequence

from . import _native
from ._native import TTCError, Tuning, check, i32, i64, lib

# TTC's --dataType letters and their element types
ELEM_BYTES = {"s": 4, "d": 8, "c": 8, "z": 16}
FLOAT_TYPES = {"s": "float", "d": "double", "c": "float complex", "z": "double complex"}
LETTER_OF_FLOAT_TYPE = {v: k for k, v in FLOAT_TYPES.items()}
VALID_DTYPES = ("s", "d", "c", "z", "sd", "ds", "cz", "zc")


def split_dtype(dtype: str):
    if dtype not in VALID_DTYPES:
        raise TTCError(5, "unknown precision. It needs to be either of the following s, d, c, z, sd, ds, cz, or zc.")
    return (dtype[0], dtype[1]) if len(dtype) == 2 else (dtype, dtype)


def torch_letter(t) -> str:
    import torch
    m = {torch.float32: "s", torch.float64: "d", torch.complex64: "c", torch.complex128: "z"}
    if t.dtype not in m:
        raise TTCError(5, f"unsupported tensor dtype {t.dtype}")
    return m[t.dtype]


def pack_scalar(letter: str, value) -> ctypes.Array:
    """alpha/beta in the precision of A (alpha) or B (beta): float, double, {float,float}, {double,double}."""
    v = complex(value)
    if letter == "s":
        if v.imag != 0:
            raise TTCError(1, "a complex scalar needs complex data")
        return (ctypes.c_float * 1)(v.real)
    if letter == "d":
        if v.imag != 0:
            raise TTCError(1, "a complex scalar needs complex data")
        return (ctypes.c_double * 1)(v.real)
    if letter == "c":
        return (ctypes.c_float * 2)(v.real, v.imag)
    return (ctypes.c_double * 2)(v.real, v.imag)


def _ptr(x) -> int:
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise TTCError(1, "A and B must be CUDA tensors (device pointers)")
        return x.data_ptr()
    raise TTCError(1, f"cannot take a device pointer of {type(x)}")


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class Plan:
    """A planned transposition ``B_{perm(i)} = alpha * A_i + beta * B_{perm(i)}`` (TTC conventions:
    column-major, perm[j] = A-dim that becomes B-dim j, lda/ldb are outer sizes)."""

    def __init__(self, perm: Sequence[int], size: Sequence[int], dtype: str = "s", beta_nonzero: bool = False,
                 lda: Optional[Sequence[int]] = None, ldb: Optional[Sequence[int]] = None,
                 tuning: Optional[Tuning | dict] = None):
        self.perm = [int(p) for p in perm]
        self.size = [int(s) for s in size]
        self.dtype = dtype
        self.ta, self.tb = split_dtype(dtype)
        self.beta_nonzero = bool(beta_nonzero)
        self.lda = [int(x) for x in lda] if lda else None
        self.ldb = [int(x) for x in ldb] if ldb else None
        if isinstance(tuning, dict):
            tuning = Tuning.make(**tuning)
        self.tuning = tuning
        if len(self.perm) != len(self.size):
            raise TTCError(2, "dimension of permutation and size does not match.")
        rank = len(self.size)
        self._h = ctypes.c_void_p()
        check(lib().ttcb_plan_create(
            ctypes.byref(self._h), rank, i32(self.perm), i64(self.size),
            i64(self.lda) if self.lda else None, i64(self.ldb) if self.ldb else None,
            _native.DTYPES[self.ta], _native.DTYPES[self.tb], int(self.beta_nonzero),
            ctypes.byref(tuning) if tuning is not None else None))

    @property
    def handle(self) -> int:
        return self._h.value or 0

    def __call__(self, A, B, alpha=1.0, beta=0.0, stream=None) -> None:
        """Launches the transposition on ``stream`` (default: torch's current stream). Asynchronous."""
        if self._h.value is None:
            raise TTCError(1, "plan was destroyed")
        if complex(beta) != 0 and not self.beta_nonzero:
            raise TTCError(11, "plan was created for beta == 0")
        al = pack_scalar(self.ta, alpha)
        be = pack_scalar(self.tb, beta) if self.beta_nonzero else None
        check(lib().ttcb_transpose(self._h, _ptr(A), _ptr(B), ctypes.cast(al, ctypes.c_void_p),
                                   ctypes.cast(be, ctypes.c_void_p) if be is not None else None,
                                   _stream_handle(stream)))

    def describe(self) -> dict:
        n = lib().ttcb_plan_describe(self._h, None, 0)
        buf = ctypes.create_string_buffer(n)
        lib().ttcb_plan_describe(self._h, buf, n)
        return json.loads(buf.value.decode())

    def launches(self) -> int:
        """Kernels one call launches (with 16-byte aligned tensors): see `describe_launches`."""
        return describe_launches(self.describe())

    def wait_timeouts(self) -> int:
        """Stage waits of the staged kernel's bulk-copy form that ran out of time since the last
        query (0 when every launch's copies landed); reading clears the count."""
        n = ctypes.c_uint(0)
        check(lib().ttcb_plan_wait_timeouts(self._h, ctypes.byref(n)))
        return int(n.value)

    @property
    def bytes(self) -> int:
        """Algorithmic bytes per call: N*(|TA| + |TB|*(1+[beta!=0]))."""
        return int(lib().ttcb_plan_bytes(self._h))

    def close(self) -> None:
        if self._h.value:
            lib().ttcb_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_plan_cache: dict = {}


def transpose(A, B, perm: Sequence[int], size: Optional[Sequence[int]] = None, alpha=1.0, beta=0.0,
              lda: Optional[Sequence[int]] = None, ldb: Optional[Sequence[int]] = None, stream=None,
              tuning: Optional[dict] = None) -> None:
    """``B = alpha * perm(A) + beta * B`` on CUDA tensors. ``size`` defaults to A's shape read in
    column-major order (i.e. ``reversed(A.shape)``); A and B are read as flat buffers."""
    if size is None:
        size = list(reversed(A.shape))
    dtype = torch_letter(A)
    tb = torch_letter(B)
    if tb != dtype:
        dtype = dtype + tb
    key = (tuple(perm), tuple(size), dtype, complex(beta) != 0, tuple(lda or ()), tuple(ldb or ()),
           tuple(sorted((k, tuple(v) if isinstance(v, list) else v) for k, v in (tuning or {}).items())),
           A.device.index)
    plan = _plan_cache.get(key)
    if plan is None:
        plan = Plan(perm, size, dtype, complex(beta) != 0, lda, ldb, tuning)
        _plan_cache[key] = plan
    plan(A, B, alpha, beta, stream)


def describe_launches(d: dict) -> int:
    """Kernels a call of the plan described by `d` launches: its kernel, and for a staged tile plan
    with ragged tiles either its edge plans' kernels or the element-wise ragged-tile kernel."""
    t = d.get("tile") or {}
    n = 1
    if t.get("async") and t.get("ragged_tiles", 0) > 0 and d.get("tile_variant", 0) in (0, 3):
        edges = d.get("edges") or []
        n += sum(describe_launches(e["plan"]) for e in edges) if edges else 1
    return n


def plan_host_json(perm, size, dtype="s", beta_nonzero=False, lda=None, ldb=None, tuning=None) -> dict:
    """The planner's decision for a problem, computed on the host only (no GPU needed)."""
    ta, tb = split_dtype(dtype)
    if isinstance(tuning, dict):
        tuning = Tuning.make(**tuning)
    buf = ctypes.create_string_buffer(8192)
    st = lib().ttcb_test_plan_host(len(size), i32(perm), i64(size), i64(lda) if lda else None,
                                   i64(ldb) if ldb else None, _native.DTYPES[ta], _native.DTYPES[tb],
                                   int(bool(beta_nonzero)), ctypes.byref(tuning) if tuning else None, buf, 8192)
    check(st)
    return json.loads(buf.value.decode())


def plan_shapes(perm, size, dtype="s", beta_nonzero=False, lda=None, ldb=None, tunings=()) -> list:
    """Shape-only plans (kernel, tile extents, access widths, cost estimate; no descriptor tables)
    of one problem under several tunings, in one host call. None where a tuning does not plan."""
    ta, tb = split_dtype(dtype)
    n = len(tunings)
    if n == 0:
        return []
    arr = (Tuning * n)(*[Tuning.make(**(t or {})) for t in tunings])
    args = (len(size), i32(perm), i64(size), i64(lda) if lda else None, i64(ldb) if ldb else None,
            _native.DTYPES[ta], _native.DTYPES[tb], int(bool(beta_nonzero)), arr, n)
    size_guess = 1024 * n
    buf = ctypes.create_string_buffer(size_guess)
    need = lib().ttcb_test_plan_shapes(*args, buf, size_guess)
    if need > size_guess:
        buf = ctypes.create_string_buffer(need)
        lib().ttcb_test_plan_shapes(*args, buf, need)
    return json.loads(buf.value.decode())


def fuse(perm, size, strideA, strideB):
    """The library's index fusion (host only): returns (perm, size, strideA, strideB)."""
    r = len(size)
    orank = ctypes.c_int()
    op = (ctypes.c_int * r)()
    on = (ctypes.c_int64 * r)()
    oa = (ctypes.c_int64 * r)()
    ob = (ctypes.c_int64 * r)()
    rc = lib().ttcb_test_fuse(r, i32(perm), i64(size), i64(strideA), i64(strideB), ctypes.byref(orank), op, on, oa, ob)
    if rc != 0:
        raise TTCError(2, "bad rank")
    k = orank.value
    return list(op[:k]), list(on[:k]), list(oa[:k]), list(ob[:k])
