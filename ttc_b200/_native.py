"""ctypes binding of ``libttcb200.so`` (include/ttcb200.h).

The library is built in-tree by ``ttc_b200.build``. Importing this module never falls back to
anything else: if the shared library is missing or does not load, the error is raised here.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libttcb200.so"

MAX_RANK = 10

DTYPES = {"s": 0, "d": 1, "c": 2, "z": 3}

STATUS = {
    0: "TTCB_OK", 1: "TTCB_ERR_INVALID_ARG", 2: "TTCB_ERR_RANK", 3: "TTCB_ERR_BAD_PERM", 4: "TTCB_ERR_BAD_LD",
    5: "TTCB_ERR_DTYPE", 6: "TTCB_ERR_ALIGN", 7: "TTCB_ERR_CUDA", 8: "TTCB_ERR_ALLOC", 9: "TTCB_ERR_UNSUPPORTED",
    10: "TTCB_ERR_TIMEOUT", 11: "TTCB_ERR_BETA",
}


class TTCError(RuntimeError):
    """A ttcb_status other than TTCB_OK, with the library's message."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.code = STATUS.get(status, str(status))
        super().__init__(f"[TTC] ERROR ({self.code}): {message}")


def pack_raster(order) -> tuple[int, int]:
    """An explicit loop order (the caller's dimensions, fastest-varying first) in ttcb_tuning's
    raster_lo / raster_hi encoding: 4 bits per position, holding dimension + 1."""
    order = [int(d) for d in order]
    if sorted(order) != list(range(len(order))) or not 1 <= len(order) <= MAX_RANK:
        raise TTCError(3, f"loop order {order} is not a permutation of the dimensions")
    lo = hi = 0
    for k, d in enumerate(order):
        if k < 8:
            lo |= (d + 1) << (4 * k)
        else:
            hi |= (d + 1) << (4 * (k - 8))
    return ctypes.c_int32(lo).value, hi


def unpack_raster(lo: int, hi: int) -> list:
    out = []
    for k in range(MAX_RANK):
        w = (lo & 0xFFFFFFFF) if k < 8 else hi
        d = (w >> (4 * (k % 8))) & 0xF
        if d == 0:
            break
        out.append(d - 1)
    return out


class Tuning(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int32), ("tile_elems", ctypes.c_int32), ("run_bytes", ctypes.c_int32),
                ("vec", ctypes.c_int32), ("blocks", ctypes.c_int32), ("loop_order", ctypes.c_int32),
                ("streaming", ctypes.c_int32), ("tile_variant", ctypes.c_int32), ("ragged", ctypes.c_int32),
                ("raster_lo", ctypes.c_int32), ("raster_hi", ctypes.c_int32), ("stages", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("round_robin", ctypes.c_int32),
                ("shifted_runs", ctypes.c_int32), ("bulk_copies", ctypes.c_int32),
                ("lane_map", ctypes.c_int32), ("claim_group", ctypes.c_int32)]

    @classmethod
    def make(cls, **kw) -> "Tuning":
        """Knobs by name; `raster=[d0, d1, ...]` (the caller's dimensions, fastest first) sets an
        explicit loop order (loop_order 4)."""
        t = cls()
        for k, v in kw.items():
            if k == "raster":
                t.raster_lo, t.raster_hi = pack_raster(v)
                t.loop_order = 4
            else:
                setattr(t, k, int(v))
        return t

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("raster_lo", "raster_hi")}
        if self.loop_order == 4:
            d["raster"] = unpack_raster(self.raster_lo, self.raster_hi)
        return d


_lib = None

# (name, restype, argtypes) of every symbol declared in include/ttcb200.h
_P = ctypes.c_void_p
_I64P = ctypes.POINTER(ctypes.c_int64)
_IP = ctypes.POINTER(ctypes.c_int)
PUBLIC_SYMBOLS = [
    ("ttcb_plan_create", ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, _IP, _I64P, _I64P, _I64P, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.POINTER(Tuning)]),
    ("ttcb_transpose", ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    ("ttcb_plan_destroy", None, [_P]),
    ("ttcb_plan_describe", ctypes.c_size_t, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    ("ttcb_plan_bytes", ctypes.c_int64, [_P]),
    ("ttcb_plan_wait_timeouts", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint)]),
    ("ttcb_last_error", ctypes.c_char_p, []),
    ("ttcb_version", None, [_IP, _IP, _IP]),
    ("ttcb_batch_create", ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.POINTER(_P), ctypes.POINTER(_P),
                                         ctypes.POINTER(_P), _P, _P, ctypes.c_int]),
    ("ttcb_batch_launch", ctypes.c_int, [_P, _P]),
    ("ttcb_batch_graph_launch", ctypes.c_int, [_P, _P]),
    ("ttcb_batch_status", ctypes.c_int, [_P, _P]),
    ("ttcb_batch_bytes", ctypes.c_int64, [_P]),
    ("ttcb_batch_destroy", None, [_P]),
    ("ttcb_transpose_noalloc", ctypes.c_int, [ctypes.c_int, _IP, _I64P, _I64P, _I64P, ctypes.c_int, ctypes.c_int,
                                              _P, _P, _P, _P, _P]),
]

TEST_SYMBOLS = [
    ("ttcb_test_bounded_wait", ctypes.c_int, [ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_uint)]),
    ("ttcb_test_fuse", ctypes.c_int, [ctypes.c_int, _IP, _I64P, _I64P, _I64P, _IP, _IP, _I64P, _I64P, _I64P]),
    ("ttcb_test_plan_host", ctypes.c_int, [ctypes.c_int, _IP, _I64P, _I64P, _I64P, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(Tuning), ctypes.c_char_p, ctypes.c_size_t]),
    ("ttcb_test_plan_desc", ctypes.c_size_t, [_P, _P, ctypes.c_size_t]),
    ("ttcb_test_fastdiv", ctypes.c_uint32, [ctypes.c_uint32, ctypes.c_uint32]),
    ("ttcb_test_plan_host_desc", ctypes.c_size_t, [ctypes.c_int, _IP, _I64P, _I64P, _I64P, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_int, ctypes.POINTER(Tuning), _IP, _P, ctypes.c_size_t]),
    ("ttcb_test_desc_layout", None, [_I64P]),
    ("ttcb_test_plan_shapes", ctypes.c_size_t, [ctypes.c_int, _IP, _I64P, _I64P, _I64P, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.POINTER(Tuning), ctypes.c_int, ctypes.c_char_p,
                                                ctypes.c_size_t]),
    ("ttcb_test_noalloc_limit", ctypes.c_size_t, [ctypes.c_size_t]),
    ("ttcb_test_plan_edges", ctypes.c_size_t, [ctypes.c_int, _IP, _I64P, _I64P, _I64P, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.POINTER(Tuning), ctypes.c_char_p, ctypes.c_size_t]),
]


def lib() -> ctypes.CDLL:
    """Loads libttcb200.so (raises if it is missing; there is no other implementation)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ttc_b200.build` "
                              "(the transposition has no non-CUDA fallback)")
        l = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | ctypes.RTLD_GLOBAL)
        for name, res, args in PUBLIC_SYMBOLS + TEST_SYMBOLS:
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def last_error() -> str:
    return lib().ttcb_last_error().decode(errors="replace")


def check(status: int) -> None:
    if status != 0:
        raise TTCError(status, last_error())


def i64(vals):
    return (ctypes.c_int64 * len(vals))(*[int(v) for v in vals])


def i32(vals):
    return (ctypes.c_int * len(vals))(*[int(v) for v in vals])
