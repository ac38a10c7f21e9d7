"""TEST INFRASTRUCTURE - runner for TTC's own generated CPU code (the timed CPU baseline).

``oracle/make_ref.py`` (run where the TTC sources are available) generates, with TTC's own search,
the AVX C++ transposition for a sample of the sweep cases and compiles it into
``oracle/_ref/libttc_ref.so`` plus a manifest. ``available()`` returns a callable that runs the
matching generated function for a case, or None when the library was not built.
"""
from __future__ import annotations

import ctypes
import json
from pathlib import Path

import numpy as np

REF_DIR = Path(__file__).resolve().parent / "_ref"
_cache = {}


def aligned(n: int, dtype, align: int = 64) -> np.ndarray:
    """A 1-D array whose data starts on an `align`-byte boundary. TTC's generated AVX code uses
    aligned vector loads and stores (its default --align), so its buffers must be 32-byte aligned."""
    dt = np.dtype(dtype)
    raw = np.empty(n * dt.itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * dt.itemsize].view(dt)


def manifest():
    f = REF_DIR / "manifest.json"
    if not f.exists():
        return None
    return json.loads(f.read_text())


def _key(c):
    return f"{c['dtype']}|{','.join(map(str, c['perm']))}|{','.join(map(str, c['size']))}|{int(c['beta'] != 0)}"


def available():
    m = manifest()
    lib_path = REF_DIR / "libttc_ref.so"
    if not m or not lib_path.exists():
        return None
    if "lib" not in _cache:
        _cache["lib"] = ctypes.CDLL(str(lib_path))
    lib = _cache["lib"]
    entries = {e["key"]: e for e in m["entries"]}

    def run(c, A: np.ndarray, B: np.ndarray, threads: int):
        if A.ctypes.data % 32 or B.ctypes.data % 32:
            raise ValueError("TTC's generated code needs 32-byte aligned buffers (use cpu_ref.aligned)")
        e = entries.get(_key(c))
        if e is None:
            raise KeyError(f"no generated TTC code for {_key(c)}")
        f = getattr(lib, e["symbol"])
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        rc = f(A.ctypes.data_as(ctypes.c_void_p), B.ctypes.data_as(ctypes.c_void_p), float(c["alpha"]),
               float(c["beta"]), int(threads))
        if rc != 0:
            raise RuntimeError(f"generated TTC code failed for {_key(c)}")
        return B

    run.keys = set(entries)
    return run
