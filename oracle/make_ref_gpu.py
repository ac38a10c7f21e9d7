"""TEST INFRASTRUCTURE - builds TTC's own CUDA transposition kernels for the B200 (reference GPU arm).

Recipe (runs where the TTC sources are: `python -m oracle.make_ref_gpu [TTC_SOURCE_DIR]`):
  1. import TTC's CUDA generator (GPUtransposeGenerator.py, CUDAtranspose.py, converted to Python 3
     by ttc_b200/py2compat.py);
  2. for each case of the 64-case sweep, fuse its indices with TTC's fuseIndices (ttc_util.py:214-276)
     and let the generator enumerate its variants the way `ttc --architecture=cuda` does
     (GPUtransposeGenerator.py:165-230, 328-349: TTC's blockings sorted by its blocking cost, every
     loop order, sorted by getCostLoop, at most --maxImplementations=200); keep the first
     VARIANTS_PER_CASE of TTC's order, the candidates its measured search would start with;
  3. emit each variant as TTC emits a measured version (GPUtransposeGenerator.getFastestVersion at
     :303-315, with the per-version names of CUDAtranspose.getHeaderName so the variants can share
     one library): its shared-memory and remainder device functions, its kernel and its host wrapper
     (CUDAtranspose.py:395-429: per-call cudaMalloc/cudaMemcpy of size/lda/ldb, launch,
     cudaDeviceSynchronize, cudaFree), one translation unit per variant;
  4. compile them with nvcc for sm_100a into oracle/_ref/libttc_ref_cuda.so and write
     oracle/_ref/cuda_manifest.json (per case: the fused sizes and leading dimensions the wrapper
     takes, and every variant's wrapper symbol, kernel name, blocking and loop order).
Nothing here runs on a GPU; oracle/cuda_ref.py loads the library and bench.py times it on the B200
(TTC's own choice among these variants is the fastest one there).
"""
from __future__ import annotations

import concurrent.futures as cf
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
REF_DIR = HERE / "_ref"
sys.path.insert(0, str(ROOT))

from ttc_b200 import py2compat as ttc_py3  # noqa: E402
from oracle.make_ref import DEFAULT_SOURCE, MAX_IMPL, case_key, sweep_cases  # noqa: E402

VARIANTS_PER_CASE = 8
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
NVCC_FLAGS = ["-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-w"]
FLOAT = {"s": "float", "d": "double"}
LIB = REF_DIR / "libttc_ref_cuda.so"
MANIFEST = REF_DIR / "cuda_manifest.json"


def variant_source(gen, impl) -> str:
    """One variant as TTC emits its measured versions: includes, the shared-memory and remainder
    device functions (only on the general path, perm[0] != 0), the kernel and the host wrapper, all
    with the variant's own names."""
    code = "#include <cuda_runtime.h>\n#include <cuComplex.h>\n#include <stdio.h>\n\n"
    if gen.perm[0] != 0:
        code += impl.getSharedTransposeKernel()
        code += impl.getRemainderTransposeKernel(32)
    code += impl.getCudaImplementation(0)
    code += impl.getHostCall(0)
    return code


def build(ttc_root: str | None = None, count: int = 64, per_case: int = VARIANTS_PER_CASE, log=print) -> Path:
    ttc_root = ttc_root or DEFAULT_SOURCE
    mods, work = ttc_py3.load(Path(ttc_root) / "ttc", ["ttc_util", "GPUreference", "CUDAtranspose",
                                                       "GPUtransposeGenerator"])
    gtg, tu = mods["GPUtransposeGenerator"], mods["ttc_util"]
    src_dir = REF_DIR / "cuda_src"
    if src_dir.exists():
        shutil.rmtree(src_dir)
    src_dir.mkdir(parents=True)
    entries, units, seen = [], [], set()
    tmp = tempfile.mkdtemp(prefix="ttc_cuda_gen_")
    for k, c in enumerate(sweep_cases(count)):
        key = case_key(c)
        if key in seen:
            continue
        seen.add(key)
        size, perm, lda, ldb = list(c["size"]), list(c["perm"]), [], []
        tu.fuseIndices(size, perm, [], lda, ldb)
        lda = list(size)  # dense: TTC's generator fills the defaults from the fused sizes
        ldb = [size[p] for p in perm]
        ft = FLOAT[c["dtype"]]
        gen = gtg.GPUtransposeGenerator(perm, [], size, float(c["alpha"]), float(c["beta"]), MAX_IMPL, ft, ft, [],
                                        1, [], list(lda), list(ldb), tmp)
        gen.getSolutions()
        variants = []
        for j, impl in enumerate(gen.implementations[:per_case]):
            name = impl.getHeaderName(0, 0)
            f = src_dir / f"case{k}_v{j}.cu"
            f.write_text(variant_source(gen, impl))
            units.append(f)
            variants.append({"symbol": name, "kernel": impl.getHeaderName(1, 0), "version": impl.getVersionName(),
                             "blocking": list(impl.blocking), "loop_perm": list(impl.loopPerm),
                             "threads": impl.vectorLength})
        entries.append({"key": key, "case": k, "size": size, "perm": perm, "lda": lda, "ldb": ldb,
                        "dtype": c["dtype"], "beta_nonzero": int(c["beta"] != 0),
                        "candidates": len(gen.implementations), "variants": variants})
        log(f"[make_ref_gpu] case {k}: {len(variants)} of {len(gen.implementations)} variants, first "
            f"{variants[0]['version'] if variants else '-'}")
    ttc_py3.cleanup(work)
    shutil.rmtree(tmp, ignore_errors=True)

    obj_dir = REF_DIR / "cuda_obj"
    obj_dir.mkdir(exist_ok=True)

    def compile_one(f: Path) -> str:
        obj = obj_dir / (f.stem + ".o")
        r = subprocess.run([NVCC, *NVCC_FLAGS, "-c", str(f), "-o", str(obj)], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {f.name}: {r.stderr[-2000:]}")
        return str(obj)

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(compile_one, units))
    out_tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([NVCC, "-shared", *NVCC_FLAGS[1:3], "-o", str(out_tmp), *objs, "-cudart", "static"], check=True)
    os.replace(out_tmp, LIB)
    MANIFEST.write_text(json.dumps({"max_implementations": MAX_IMPL, "variants_per_case": per_case,
                                    "nvcc_flags": NVCC_FLAGS, "entries": entries}, indent=1))
    return LIB


def build_if_missing(ttc_root: str | None = None):
    if LIB.exists() and MANIFEST.exists():
        return LIB
    return build(ttc_root)


if __name__ == "__main__":
    a = [x for x in sys.argv[1:] if not x.startswith("--")]
    print(build(a[0] if a else None))
