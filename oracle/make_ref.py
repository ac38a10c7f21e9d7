"""TEST INFRASTRUCTURE - builds oracle/_ref/: TTC's own generated CPU code for the timed baseline.

Recipe (runs where the TTC sources are: `python -m oracle.make_ref [TTC_SOURCE_DIR] [--count N]`,
the directory defaulting to $TTC_REFERENCE_DIR, else the reference checkout of this machine):
  1. convert the TTC package to Python 3 in a scratch directory (ttc_b200/py2compat.py);
  2. for each case of the 64-case sweep (the workload bench.py times), run TTC's own driver
     `ttc.main()` with `--architecture=avx --compiler=g++` and its default `--maxImplementations=200`:
     TTC generates its AVX variants, compiles them with its Makefile (g++ -O3 -fopenmp -march=native),
     measures them on this host and writes the fastest to ttc_transpositions/<name>.h. Each finished
     case is recorded in oracle/_ref/manifest.json at once, so an interrupted run resumes;
  3. write one small C++ file per case whose extern "C" entry calls the generated template function
     with the case's fused sizes and TTC's lda/ldb arrays, and compile them into
     oracle/_ref/libttc_ref.so with portable flags (-O3 -fopenmp -mavx2 -mfma), so the library loads
     on any x86-64 host with AVX2. oracle/cpu_ref.py recompiles the same files with TTC's own flags
     for the host it runs on (-march=native) before the baseline is timed there.
The output directory is not committed; it travels with the working tree to the GPU box, where
bench.py times it on that host's cores.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
REF_DIR = HERE / "_ref"
sys.path.insert(0, str(ROOT))

from ttc_b200 import py2compat as ttc_py3  # noqa: E402

# Where this recipe reads the TTC sources unless told otherwise.
DEFAULT_SOURCE = os.environ.get("TTC_REFERENCE_DIR", "/root/reference")

PACKAGE = ["ttc", "ttc_util", "sql_util", "transpose", "transposeGenerator", "GPUtransposeGenerator",
           "CUDAtranspose", "GPUreference"]
CTYPE = {"s": "float", "d": "double"}
MAX_IMPL = 200  # TTC's default --maxImplementations (ttc.py:1143-1175)
PORTABLE_FLAGS = ["-O3", "-fopenmp", "-mavx2", "-mfma", "-Wno-attributes"]
TTC_FLAGS = ["-O3", "-fopenmp", "-march=native", "-Wno-attributes"]  # TTC's Makefile, target g++


def sweep_cases(count: int):
    import ttc_b200.workloads as wl
    return wl.sweep_cases(2024)[:count]


def case_key(c):
    return f"{c['dtype']}|{','.join(map(str, c['perm']))}|{','.join(map(str, c['size']))}|{int(c['beta'] != 0)}"


def _manifest_path():
    return REF_DIR / "manifest.json"


def load_manifest() -> dict:
    f = _manifest_path()
    if f.exists():
        return json.loads(f.read_text())
    return {"max_implementations": MAX_IMPL, "entries": []}


def case_source(entry: dict, c: dict) -> str:
    """C++ source of one case's extern "C" entry point around TTC's generated function."""
    from ttc_b200.ttc_util import denseLeadingDims, fuseIndices
    t = CTYPE[c["dtype"]]
    # TTC fuses indices before generating, so the template arguments are the fused extents; the
    # dense leading dimensions follow from the fused sizes
    fsize, fperm, flda, fldb = list(c["size"]), list(c["perm"]), [], []
    fuseIndices(fsize, fperm, [], flda, fldb)
    flda, fldb = denseLeadingDims(fsize, fperm, flda, fldb)
    call_beta = f", ({t})beta" if c["beta"] != 0 else ""
    return ("#include <omp.h>\n#include \"ttc_offset.h\"\n"
            f"#include \"{entry['header']}\"\n"
            f'extern "C" int {entry["symbol"]}(const void* A, void* B, double alpha, double beta, int threads) {{\n'
            f"  const int lda[] = {{{', '.join(map(str, flda))}}};\n"
            f"  const int ldb[] = {{{', '.join(map(str, fldb))}}};\n"
            f"  if (threads > 0) omp_set_num_threads(threads);\n"
            f"  {entry['function']}<{', '.join(map(str, fsize))}>((const {t}*)A, ({t}*)B, ({t})alpha{call_beta}, "
            f"lda, ldb);\n  return 0;\n}}\n")


def compile_library(src_dir: Path, entries: list, out: Path, flags: list, jobs: int | None = None) -> Path:
    """Compiles one object per case (in parallel) from src_dir/case_<k>.cpp and links `out`."""
    import concurrent.futures as cf
    obj_dir = out.parent / (out.stem + "_obj")
    obj_dir.mkdir(parents=True, exist_ok=True)

    def one(e):
        src = src_dir / f"case_{e['case']}.cpp"
        obj = obj_dir / f"case_{e['case']}.o"
        subprocess.run(["g++", *flags, "-fPIC", "-I", str(src_dir), "-c", str(src), "-o", str(obj)], check=True,
                       capture_output=True)
        return str(obj)

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(one, entries))
    tmp = out.with_suffix(".so.tmp")
    subprocess.run(["g++", "-shared", "-fopenmp", "-o", str(tmp), *objs], check=True, capture_output=True)
    os.replace(tmp, out)
    return out


def build(ttc_root: str | None = None, count: int = 64, max_impl: int = MAX_IMPL, threads: int | None = None,
          log=print, max_seconds: float | None = None) -> Path:
    """Runs TTC's search for every case not yet in the manifest (stopping, resumably, once
    `max_seconds` have passed) and compiles the library from the cases that are there."""
    t_start = time.time()
    ttc_root = ttc_root or DEFAULT_SOURCE
    threads = threads or os.cpu_count() or 1
    REF_DIR.mkdir(exist_ok=True)
    man = load_manifest()
    if man.get("max_implementations") != max_impl:
        man = {"max_implementations": max_impl, "entries": []}
    man["threads_at_tuning"] = threads
    man["tuning_flags"] = TTC_FLAGS
    have = {e["key"] for e in man["entries"]}
    cases = sweep_cases(count)
    todo = [(k, c) for k, c in enumerate(cases) if case_key(c) not in have]
    if todo:
        work = Path(tempfile.mkdtemp(prefix="ttc_ref_build_"))
        pkg = work / "ttc"
        ttc_py3.convert_tree(Path(ttc_root) / "ttc", pkg, PACKAGE)
        (pkg / "__init__.py").write_text("from . import ttc\n")
        env = dict(os.environ, TTC_ROOT=str(work))
        env.pop("CC", None)
        env.pop("CXX", None)
        for k, c in todo:
            if max_seconds is not None and time.time() - t_start > max_seconds:
                log(f"[make_ref] stopping after {max_seconds:.0f} s; {len(man['entries'])} cases searched")
                break
            run_dir = work / f"run{k}"
            run_dir.mkdir()
            args = [f"--perm={','.join(map(str, c['perm']))}", f"--size={','.join(map(str, c['size']))}",
                    f"--dataType={c['dtype']}", f"--alpha={c['alpha']}", f"--beta={c['beta']}",
                    f"--numThreads={threads}", "--compiler=g++", "--architecture=avx",
                    f"--affinity=0-{threads - 1}", f"--maxImplementations={max_impl}", "--ignoreDatabase"]
            code = ("import sys; sys.path.insert(0, %r); sys.argv = ['ttc'] + %r; "
                    "from ttc.ttc import main; main()" % (str(work), args))
            t0 = time.time()
            r = subprocess.run([sys.executable, "-c", code], cwd=run_dir, env=env, capture_output=True, text=True)
            out_dir = run_dir / "ttc_transpositions"
            found = [h for h in sorted(out_dir.glob("*.h")) if h.name != "ttc_offset.h"] if out_dir.exists() else []
            if r.returncode != 0 or not found:
                raise RuntimeError(f"TTC failed for case {k}: {r.stdout[-2000:]}\n{r.stderr[-2000:]}")
            header = f"case_{k}_{found[0].name}"
            shutil.copy(found[0], REF_DIR / header)
            if not (REF_DIR / "ttc_offset.h").exists():
                shutil.copy(out_dir / "ttc_offset.h", REF_DIR / "ttc_offset.h")
            fastest = [ln for ln in r.stdout.splitlines() if "fastest version" in ln.lower()]
            impl = [ln for ln in r.stdout.splitlines() if "implementations done" in ln]
            entry = {"key": case_key(c), "case": k, "function": found[0].stem, "header": header,
                     "symbol": f"ttc_ref_case{k}", "ttc_report": fastest[-1].strip() if fastest else "",
                     "implementations": impl[-1].split("out of")[-1].split("impl")[0].strip() if impl else "",
                     "search_seconds": round(time.time() - t0, 1)}
            man["entries"] = [e for e in man["entries"] if e["key"] != entry["key"]] + [entry]
            man["entries"].sort(key=lambda e: e["case"])
            _manifest_path().write_text(json.dumps(man, indent=1))
            log(f"[make_ref] case {k}: {entry['ttc_report']} ({entry['search_seconds']} s)")
            shutil.rmtree(run_dir, ignore_errors=True)
        shutil.rmtree(work, ignore_errors=True)
    by_key = {case_key(c): c for c in cases}
    for e in man["entries"]:
        (REF_DIR / f"case_{e['case']}.cpp").write_text(case_source(e, by_key[e["key"]]))
    lib = compile_library(REF_DIR, man["entries"], REF_DIR / "libttc_ref.so", PORTABLE_FLAGS)
    man["library_flags"] = PORTABLE_FLAGS
    _manifest_path().write_text(json.dumps(man, indent=1))
    return lib


def build_if_missing(ttc_root: str | None = None, count: int = 64, max_seconds: float | None = None):
    man = load_manifest()
    need = {case_key(c) for c in sweep_cases(count)}
    if (REF_DIR / "libttc_ref.so").exists() and need <= {e["key"] for e in man["entries"]} and \
            man.get("max_implementations") == MAX_IMPL and man.get("library_flags") == PORTABLE_FLAGS:
        return REF_DIR / "libttc_ref.so"
    return build(ttc_root, count=count, max_seconds=max_seconds)


if __name__ == "__main__":
    a = [x for x in sys.argv[1:] if not x.startswith("--")]
    n = 64
    for x in sys.argv[1:]:
        if x.startswith("--count="):
            n = int(x.split("=", 1)[1])
    print(build(a[0] if a else None, count=n))
