"""Generates tests/golden/ttc_reference_loop.npz: outputs of TTC's own reference transposition.

TTC's correctness oracle is a C++ loop nest that its GPU generator emits for every transposition
(GPUreference.referenceTranspose, GPUreference.py:33-244 in the TTC project). This script imports
that generator from the TTC sources (converted to Python 3 by ttc_b200/py2compat.py), emits the loop for each
case of TTC's own test matrix (test-framework/ttc_test.py:80-92, first size of every permutation,
every dtype pair and beta of the sweep) plus padded lda/ldb cases, compiles all of them into one
host program with g++ (cuComplex.h from the CUDA toolkit for the complex types, no -march, so no
fused multiply-add exists), runs it on seeded uniform[-1, 1] inputs and stores the results.

Run in a container that has the TTC sources (path as the first argument); the fixture is what the
tests read. Inputs are not stored: the tests regenerate them from the seeds and check their SHA-256.
"""
from __future__ import annotations

import hashlib
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

import helpers  # noqa: E402
from ttc_b200 import py2compat as ttc_py3  # noqa: E402

OUT = HERE / "ttc_reference_loop.npz"
CU_TYPES = {"s": "float", "d": "double", "c": "cuFloatComplex", "z": "cuDoubleComplex"}
REAL_TYPES = {"s": "float", "d": "double", "c": "float", "z": "double"}


def golden_cases():
    cases = []
    seed = 1000
    for c, perm in enumerate(helpers.TTC_PERMS):
        size = helpers.TTC_SIZES[c][0]
        for dtype in helpers.TTC_DTYPES:
            for beta in helpers.TTC_BETAS:
                cases.append(dict(perm=perm, size=size, dtype=dtype, alpha=1.1, beta=float(beta), lda=None,
                                  ldb=None, seed=seed))
                seed += 2
    # sub-tensors (lda/ldb padding), including the strided configuration's permutation
    padded = [([3, 1, 0, 2], [9, 8, 7, 6], [13, 8, 9, 6], None),
              ([2, 0, 3, 1], [7, 5, 4, 6], [9, 6, 4, 7], [4, 8, 7, 5]),
              ([1, 2, 0], [13, 7, 5], None, [7, 8, 13]),
              ([1, 0], [17, 23], [20, 23], [25, 17])]
    for perm, size, lda, ldb in padded:
        for dtype in helpers.TTC_DTYPES:
            for beta in (0.0, -0.5):
                cases.append(dict(perm=perm, size=size, dtype=dtype, alpha=1.5, beta=beta, lda=lda, ldb=ldb,
                                  seed=seed))
                seed += 2
    return cases


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(a.tobytes()).hexdigest()


def main(ttc_root: str):
    mods, work = ttc_py3.load(Path(ttc_root) / "ttc", ["ttc_util", "GPUreference"])
    GPUreference = mods["GPUreference"]
    cases = golden_cases()
    funcs = {}
    calls = []
    blob = bytearray()
    layout = []
    for k, c in enumerate(cases):
        ta, tb = helpers.split(c["dtype"])
        rank = len(c["size"])
        lda = c["lda"] or list(c["size"])
        ldb = c["ldb"] or [c["size"][p] for p in c["perm"]]
        ref = GPUreference.referenceTranspose(c["perm"], list(range(rank))[::-1], c["size"], c["alpha"], c["beta"],
                                              CU_TYPES[ta], CU_TYPES[tb], lda, ldb)
        name = ref.getReferenceHeader()
        if name not in funcs:
            funcs[name] = ref.generateReferenceImplementation()
        A, B = helpers.make_inputs(c["size"], c["perm"], c["dtype"], c["seed"], c["lda"], c["ldb"])
        c["sha_A"], c["sha_B"] = sha(A), sha(B)
        offA = len(blob)
        blob += A.tobytes()
        blob += b"\0" * (-len(blob) % 16)
        offB = len(blob)
        blob += B.tobytes()
        blob += b"\0" * (-len(blob) % 16)
        layout.append((offA, offB, B.size, B.dtype))
        talpha = "double" if ta in "dz" else "float"
        tbeta = "double" if tb in "dz" else "float"
        sz = ",".join(str(x) for x in c["size"])
        la = ",".join(str(x) for x in lda)
        lb = ",".join(str(x) for x in ldb)
        args = f"(const {CU_TYPES[ta]}*)(in + {offA}), ({CU_TYPES[tb]}*)(out + {offB}), size{k}, ({talpha}){c['alpha']!r}"
        if c["beta"] != 0:
            args += f", ({tbeta}){c['beta']!r}"
        args += f", lda{k}, ldb{k}"
        calls.append(f"  {{ int size{k}[] = {{{sz}}}; int lda{k}[] = {{{la}}}; int ldb{k}[] = {{{lb}}};\n"
                     f"    {name}({args}); }}\n")
    src = "#include <cstdio>\n#include <cstdlib>\n#include <cstring>\n#include <omp.h>\n#include <cuComplex.h>\n\n"
    src += "\n".join(funcs.values())
    src += ("\nint main(int argc, char** argv) {\n"
            "  FILE* f = fopen(argv[1], \"rb\"); fseek(f, 0, SEEK_END); long n = ftell(f); fseek(f, 0, SEEK_SET);\n"
            "  char* in = (char*)malloc(n); char* out = (char*)malloc(n);\n"
            "  if (fread(in, 1, n, f) != (size_t)n) return 1; fclose(f); memcpy(out, in, n);\n")
    src += "".join(calls)
    src += "  f = fopen(argv[2], \"wb\"); fwrite(out, 1, n, f); fclose(f); return 0;\n}\n"
    tmp = Path(tempfile.mkdtemp(prefix="ttc_golden_"))
    (tmp / "golden.cpp").write_text(src)
    (tmp / "in.bin").write_bytes(bytes(blob))
    subprocess.run(["g++", "-O2", "-fopenmp", "-I/usr/local/cuda/include", "-o", str(tmp / "golden"),
                    str(tmp / "golden.cpp")], check=True)
    subprocess.run([str(tmp / "golden"), str(tmp / "in.bin"), str(tmp / "out.bin")], check=True)
    out = (tmp / "out.bin").read_bytes()
    arrays = {}
    for k, (offA, offB, nb, dt) in enumerate(layout):
        arrays[f"B{k}"] = np.frombuffer(out, dtype=dt, count=nb, offset=offB).copy()
    meta = json.dumps({"generator": "TTC GPUreference.referenceTranspose, compiled with g++ -O2 -fopenmp",
                       "cases": cases})
    np.savez_compressed(OUT, meta=np.frombuffer(meta.encode(), dtype=np.uint8), **arrays)
    ttc_py3.cleanup(work)
    print(f"wrote {OUT} with {len(cases)} cases ({OUT.stat().st_size / 1e6:.2f} MB)")


if __name__ == "__main__":
    from oracle.make_ref import DEFAULT_SOURCE
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SOURCE)
