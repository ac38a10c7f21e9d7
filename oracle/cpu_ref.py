"""TEST INFRASTRUCTURE - runner for TTC's own generated CPU code (the timed CPU baseline).

``oracle/make_ref.py`` (run where the TTC sources are available) generates, with TTC's own search,
the AVX C++ transposition for every case of the 64-case sweep and compiles it into
``oracle/_ref/libttc_ref.so`` (portable AVX2 flags) plus a manifest and one C++ file per case.
``available()`` returns a callable that runs the matching generated function for a case, or None
when the library was not built. ``available(native=True)`` first recompiles the same files with
TTC's own Makefile flags for the host it runs on (g++ -O3 -fopenmp -march=native), which is how
the benchmark times it on the GPU box's cores.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import platform
import time
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


def host_id() -> str:
    """The CPU model of this host (the -march=native build is specific to it)."""
    model = platform.processor() or ""
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model


def native_library() -> tuple[Path, float]:
    """Compiles the generated cases with TTC's own flags for this host (once per host model);
    returns the library path and the seconds the compile took (0 when it was already there)."""
    from oracle import make_ref
    m = manifest()
    tag = hashlib.sha256((host_id() + json.dumps(m["entries"], sort_keys=True)).encode()).hexdigest()[:12]
    out = REF_DIR / "host" / f"libttc_ref_{tag}.so"
    if out.exists():
        return out, 0.0
    out.parent.mkdir(parents=True, exist_ok=True)
    t0 = time.perf_counter()
    make_ref.compile_library(REF_DIR, m["entries"], out, make_ref.TTC_FLAGS)
    return out, time.perf_counter() - t0


def available(native: bool = False):
    m = manifest()
    lib_path = REF_DIR / "libttc_ref.so"
    if not m or not lib_path.exists() or not all("symbol" in e for e in m.get("entries", [])):
        return None
    compile_s = 0.0
    if native:
        lib_path, compile_s = native_library()
    key = str(lib_path)
    if key not in _cache:
        _cache[key] = ctypes.CDLL(str(lib_path))
    lib = _cache[key]
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
    run.library = str(lib_path)
    run.flags = " ".join(make_flags(native))
    run.compile_seconds = compile_s
    run.max_implementations = m.get("max_implementations")
    run.threads_at_tuning = m.get("threads_at_tuning")
    run.entries = entries
    return run


def make_flags(native: bool):
    from oracle import make_ref
    return make_ref.TTC_FLAGS if native else make_ref.PORTABLE_FLAGS
