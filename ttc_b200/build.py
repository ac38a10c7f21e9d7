"""Builds ``ttc_b200/libttcb200.so`` (the C ABI over the sm_100a kernels) with nvcc.

Sources are compiled in parallel into ``_build/`` and linked in-tree, so the shared library travels
with the source tree. Usage: ``python -m ttc_b200.build [--force]``.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libttcb200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-I", str(ROOT / "include")]

PAIRS = ["ss", "dd", "cc", "zz", "sd", "ds", "cz", "zc"]


def _units():
    units = []
    for i, name in enumerate(PAIRS):
        units.append((CSRC / "kernels_pair.cu", BUILD / f"kernels_{name}.o", [f"-DTTCB_PAIR={i}"]))
    for src in ("abi.cu", "batched.cu", "noalloc.cu", "mlp.cu"):
        if (CSRC / src).exists():
            units.append((CSRC / src, BUILD / (Path(src).stem + ".o"), []))
    units.append((CSRC / "plan.cpp", BUILD / "plan.o", ["-x", "cu"]))
    return units


def _fingerprint(extra: list[str]) -> str:
    h = hashlib.sha256()
    for p in sorted(CSRC.iterdir()):
        if p.suffix in (".cu", ".cuh", ".h", ".cpp"):
            h.update(p.name.encode())
            h.update(p.read_bytes())
    for hdr in sorted((ROOT / "include").glob("*.h")):
        h.update(hdr.read_bytes())
    h.update(" ".join(ARCH + COMMON + extra).encode())
    return h.hexdigest()


def _compile(unit):
    src, obj, flags = unit
    cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every CUDA/C++ source for sm_100a and links libttcb200.so. Returns its path."""
    BUILD.mkdir(exist_ok=True)
    stamp = BUILD / "libttcb200.stamp"
    fp = _fingerprint([])
    if not force and LIB.exists() and stamp.exists() and stamp.read_text() == fp:
        return LIB
    units = _units()
    with cf.ThreadPoolExecutor(max_workers=min(len(units), os.cpu_count() or 4)) as ex:
        results = list(ex.map(_compile, units))
    if verbose:
        for obj, err in results:
            if err.strip():
                print(f"[{obj.name}] {err}", file=sys.stderr)
    objs = [str(o) for o, _ in results]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *objs, "-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    stamp.write_text(fp)
    return LIB


if __name__ == "__main__":
    t = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(t)
