"""TEST INFRASTRUCTURE - runner for TTC's own CUDA transposition kernels (the reference GPU arm).

``oracle/make_ref_gpu.py`` (run where the TTC sources are) emits, with TTC's CUDA generator, the first
variants of TTC's own ordering for every case of the 64-case sweep and compiles them for sm_100a
into ``oracle/_ref/libttc_ref_cuda.so``. ``available()`` returns a ``CudaReference`` over that
library, or None when it was not built. A variant is called through TTC's generated host wrapper
(CUDAtranspose.py:395-429 in the TTC project): it copies the fused sizes and leading dimensions to
freshly allocated device buffers, launches the kernel, synchronizes the device and frees them.
"""
from __future__ import annotations

import ctypes
import json
from pathlib import Path

REF_DIR = Path(__file__).resolve().parent / "_ref"
LIB = REF_DIR / "libttc_ref_cuda.so"
MANIFEST = REF_DIR / "cuda_manifest.json"


def _key(c):
    return f"{c['dtype']}|{','.join(map(str, c['perm']))}|{','.join(map(str, c['size']))}|{int(c['beta'] != 0)}"


class CudaReference:
    def __init__(self):
        self.lib = ctypes.CDLL(str(LIB))
        m = json.loads(MANIFEST.read_text())
        self.manifest = m
        self.entries = {e["key"]: e for e in m["entries"]}

    def covers(self, c) -> bool:
        return _key(c) in self.entries

    def variants(self, c) -> list:
        return self.entries[_key(c)]["variants"]

    def call(self, c, variant: int, A_ptr: int, B_ptr: int):
        """One call of TTC's wrapper for variant `variant` of case `c` on device pointers (synchronous,
        like TTC's wrapper)."""
        e = self.entries[_key(c)]
        v = e["variants"][variant]
        f = getattr(self.lib, v["symbol"])
        real = ctypes.c_float if e["dtype"] == "s" else ctypes.c_double
        ints = lambda xs: (ctypes.c_int * len(xs))(*[int(x) for x in xs])
        args = [ctypes.c_void_p(A_ptr), ctypes.c_void_p(B_ptr), real(float(c["alpha"]))]
        if e["beta_nonzero"]:
            args.append(real(float(c["beta"])))
        args += [ints(e["size"]), ints(e["lda"]), ints(e["ldb"])]
        f.restype = None
        f(*args)


def available():
    if not LIB.exists() or not MANIFEST.exists():
        return None
    return CudaReference()
