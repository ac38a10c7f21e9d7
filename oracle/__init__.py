"""TEST INFRASTRUCTURE - the CPU oracle of the transposition.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this package, and only as the checker or the timed CPU baseline; the product path never does.

``transpose()`` wraps ``ttc_oracle.c``: a C restatement of the scalar reference loop that TTC
generates (GPUreference.py:33-244 in the TTC project), compiled without floating-point
contraction. ``ttc_ref`` restates TTC's index fusion and loop-order cost heuristic in Python.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libttc_oracle.so"

DTYPE_CODES = {"s": 0, "d": 1, "c": 2, "z": 3}
NUMPY_TYPES = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}

_lib = None


def build() -> Path:
    """Compiles the oracle with the Makefile next to it (gcc, -ffp-contract=off, OpenMP)."""
    src = HERE / "ttc_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        env = dict(os.environ)
        env.pop("CFLAGS", None)
        subprocess.run(["make", "-C", str(HERE), "-s"], check=True, env=env)
    return LIB


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        args = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int64),
                ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64), ctypes.c_int, ctypes.c_int,
                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                ctypes.c_void_p, ctypes.c_void_p]
        lib.ttco_transpose.argtypes = args
        lib.ttco_transpose.restype = ctypes.c_int
        lib.ttco_transpose_par.argtypes = args + [ctypes.c_int]
        lib.ttco_transpose_par.restype = ctypes.c_int
        _lib = lib
    return _lib


def _arr(vals, ctype):
    if vals is None:
        return None
    return (ctype * len(vals))(*[int(v) for v in vals])


def transpose(A: np.ndarray, B: np.ndarray, perm, size, alpha=1.0, beta=0.0, lda=None, ldb=None,
              dtype: str = "s", threads: int = 0) -> np.ndarray:
    """In-place ``B = alpha * perm(A) + beta * B`` on flat numpy buffers (TTC conventions).

    ``dtype`` is TTC's --dataType letter pair ('s', 'd', 'c', 'z', 'sd', 'ds', 'cz', 'zc').
    ``alpha``/``beta`` may be complex (the imaginary part is used for complex types only).
    ``threads`` > 0 runs the OpenMP form. Returns B.
    """
    lib = _load()
    ta, tb = (dtype[0], dtype[1]) if len(dtype) == 2 else (dtype, dtype)
    assert A.dtype == NUMPY_TYPES[ta] and B.dtype == NUMPY_TYPES[tb], (A.dtype, B.dtype, dtype)
    assert A.flags.c_contiguous and B.flags.c_contiguous
    rank = len(size)
    from .ttc_ref import strides
    if all(int(x) > 0 for x in size):
        sA, sB = strides(size, perm, lda, ldb)
        need_a = sum((int(n) - 1) * s for n, s in zip(size, sA)) + 1
        need_b = sum((int(n) - 1) * s for n, s in zip(size, sB)) + 1
        if A.size < need_a or B.size < need_b:
            raise ValueError(f"buffers too small: A {A.size} < {need_a} or B {B.size} < {need_b}")
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    beta_nz = 1 if complex(beta) != 0 else 0
    args = (rank, _arr(perm, ctypes.c_int), _arr(size, ctypes.c_int64), _arr(lda, ctypes.c_int64),
            _arr(ldb, ctypes.c_int64), DTYPE_CODES[ta], DTYPE_CODES[tb], al, be, beta_nz,
            A.ctypes.data_as(ctypes.c_void_p), B.ctypes.data_as(ctypes.c_void_p))
    if threads > 0:
        rc = lib.ttco_transpose_par(*args, threads)
    else:
        rc = lib.ttco_transpose(*args)
    if rc != 0:
        raise ValueError("oracle rejected the arguments")
    return B


def extents(size, perm, lda=None, ldb=None):
    """Number of elements the flat A and B buffers need (outer sizes included)."""
    la = list(lda) if lda is not None else list(size)
    lb = list(ldb) if ldb is not None else [size[p] for p in perm]
    na = int(np.prod(la[:-1], dtype=np.int64)) * int(size[-1]) if len(size) else 1
    nb = int(np.prod(lb[:-1], dtype=np.int64)) * int(size[perm[-1]]) if len(size) else 1
    return na, nb
