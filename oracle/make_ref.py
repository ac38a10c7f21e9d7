"""TEST INFRASTRUCTURE - builds oracle/_ref/: TTC's own generated CPU code for the timed baseline.

Recipe (runs where the TTC sources are, e.g. `python -m oracle.make_ref /root/reference`):
  1. convert the TTC package to Python 3 in a scratch directory (oracle/ttc_py3.py);
  2. for each sample case of the large sweep (the cases bench.py times on the CPU), run TTC's own
     driver `ttc.main()` with `--architecture=avx --compiler=g++`: TTC generates its AVX variants,
     compiles them with its Makefile, measures them on this host and writes the fastest to
     ttc_transpositions/<name>.h;
  3. compile one shared library, oracle/_ref/libttc_ref.so, whose extern "C" entry per case calls the
     generated template function with the case's sizes and TTC's lda/ldb arrays, with the number of
     OpenMP threads given at run time; write oracle/_ref/manifest.json.
The output directory is not committed; it travels with the working tree to the GPU box, where
bench.py times it on that host's cores (oracle/cpu_ref.py loads it).
"""
from __future__ import annotations

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

from oracle import ttc_py3  # noqa: E402

PACKAGE = ["ttc", "ttc_util", "sql_util", "transpose", "transposeGenerator", "GPUtransposeGenerator",
           "CUDAtranspose", "GPUreference"]
CTYPE = {"s": "float", "d": "double"}


def sample_cases(count: int):
    import ttc_b200.workloads as wl
    return wl.sweep_cases(2024)[:count]


def _key(c):
    return f"{c['dtype']}|{','.join(map(str, c['perm']))}|{','.join(map(str, c['size']))}|{int(c['beta'] != 0)}"


def build(ttc_root: str = "/root/reference", count: int = 6, max_impl: int = 24, threads: int | None = None):
    threads = threads or os.cpu_count() or 1
    work = Path(tempfile.mkdtemp(prefix="ttc_ref_build_"))
    pkg = work / "ttc"
    ttc_py3.convert_tree(Path(ttc_root) / "ttc", pkg, PACKAGE)
    (pkg / "__init__.py").write_text("from . import ttc\n")
    run_dir = work / "run"
    run_dir.mkdir()
    env = dict(os.environ, TTC_ROOT=str(work))
    env.pop("CC", None)
    env.pop("CXX", None)
    entries = []
    headers = []
    for k, c in enumerate(sample_cases(count)):
        args = [f"--perm={','.join(map(str, c['perm']))}", f"--size={','.join(map(str, c['size']))}",
                f"--dataType={c['dtype']}", f"--alpha={c['alpha']}", f"--beta={c['beta']}",
                f"--numThreads={threads}", "--compiler=g++", "--architecture=avx", f"--affinity=0-{threads - 1}",
                f"--maxImplementations={max_impl}", "--ignoreDatabase"]
        code = ("import sys; sys.path.insert(0, %r); sys.argv = ['ttc'] + %r; "
                "from ttc.ttc import main; main()" % (str(work), args))
        r = subprocess.run([sys.executable, "-c", code], cwd=run_dir, env=env, capture_output=True, text=True)
        out_dir = run_dir / "ttc_transpositions"
        before = set(headers)
        found = [h for h in sorted(out_dir.glob("*.h")) if h.name != "ttc_offset.h" and h.name not in before]
        if r.returncode != 0 or not found:
            raise RuntimeError(f"TTC failed for case {k}: {r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        name = found[0].stem
        headers.append(found[0].name)
        fastest = [ln for ln in r.stdout.splitlines() if "fastest version" in ln.lower()]
        entries.append({"key": _key(c), "case": k, "function": name, "symbol": f"ttc_ref_case{k}",
                        "ttc_report": fastest[-1].strip() if fastest else ""})
    # shim with one extern "C" entry per case
    src = ["#include <omp.h>", '#include "ttc_offset.h"']
    src += [f'#include "{h}"' for h in headers]
    from ttc_b200.ttc_util import fuseIndices
    for e, c in zip(entries, sample_cases(count)):
        t = CTYPE[c["dtype"]]
        # TTC fuses indices before generating, so the template arguments are the fused extents
        fsize, fperm, flda, fldb = list(c["size"]), list(c["perm"]), [], []
        fuseIndices(fsize, fperm, [], flda, fldb)
        sizes = ", ".join(map(str, fsize))
        lda = ", ".join(map(str, flda))
        ldb = ", ".join(map(str, fldb))
        call_beta = f", ({t})beta" if c["beta"] != 0 else ""
        src.append(f'extern "C" int {e["symbol"]}(const void* A, void* B, double alpha, double beta, int threads) {{\n'
                   f"  const int lda[] = {{{lda}}};\n  const int ldb[] = {{{ldb}}};\n"
                   f"  if (threads > 0) omp_set_num_threads(threads);\n"
                   f"  {e['function']}<{sizes}>((const {t}*)A, ({t}*)B, ({t})alpha{call_beta}, lda, ldb);\n"
                   f"  return 0;\n}}")
    REF_DIR.mkdir(exist_ok=True)
    shim = REF_DIR / "ttc_ref_shim.cpp"
    shim.write_text("\n".join(src) + "\n")
    inc = run_dir / "ttc_transpositions"
    subprocess.run(["g++", "-O3", "-fopenmp", "-mavx2", "-mfma", "-fPIC", "-shared", "-Wno-attributes",
                    "-I", str(inc), "-o", str(REF_DIR / "libttc_ref.so"), str(shim)], check=True)
    for h in headers + ["ttc_offset.h"]:
        shutil.copy(inc / h, REF_DIR / h)
    (REF_DIR / "manifest.json").write_text(json.dumps({"threads_at_tuning": threads, "max_implementations": max_impl,
                                                         "entries": entries}, indent=1))
    shutil.rmtree(work, ignore_errors=True)
    return REF_DIR / "libttc_ref.so"


def build_if_missing(ttc_root: str = "/root/reference"):
    if (REF_DIR / "libttc_ref.so").exists() and (REF_DIR / "manifest.json").exists():
        return REF_DIR / "libttc_ref.so"
    return build(ttc_root)


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
