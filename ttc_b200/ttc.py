"""TTC's driver and command line for the B200 transposition: `generateTransposition(TTCargs)` and
`main()` with the same flags, names and return values as TTC's (ttc.py:614-1376 in the TTC project).

Flow (ttc.py:614-1130): sanity checks -> index fusion (reported like TTC) -> validation -> tuning
database lookup -> measured search over candidate schedules (or the learned selector with --model)
-> write ttc_transpositions/<name>.{h,cu} -> store every variant in the database -> return
(transposeName, bandwidth of the fastest variant in GiB/s, TTC's unit). Errors raise TTCError
instead of exit(-1), except in main(), which prints them and exits with status 1 like TTC does.

    python -m ttc_b200.ttc --perm=1,0,2 --size=1000,768,16 --beta=1.0 --dataType=s --architecture=cuda
"""
from __future__ import annotations

import copy
import json
import os
import socket
import sys
import time
from pathlib import Path

from . import sql_util, ttc_util
from ._native import TTCError
from .ttc_util import ENDC, FAIL, OKGREEN, WARNING, TTCargs

ALLOWED = ["--compiler", "--streamingStores", "--use-streamingStores", "--maxImplementations", "--help", "--alpha",
           "--beta", "--papi", "--size", "--perm", "--loopPerm", "--floatType", "--dataType", "--numThreads",
           "--generateOnly", "--prefetchDistances", "--keep", "--updateDatabase", "--dontCompile", "-v",
           "--blockings", "--noTest", "--no-align", "--no-vec", "--mpi", "--architecture", "--affinity", "--lda",
           "--ldb", "--ignoreDatabase", "--threadsPerBlock", "--hotA", "--hotB", "--verbose",
           # additions
           "--model", "--confidence", "--batched", "--database"]

DTYPE_ARG = {"s": ("float", "float"), "d": ("double", "double"), "c": ("float complex", "float complex"),
             "z": ("double complex", "double complex"), "sd": ("float", "double"), "ds": ("double", "float"),
             "cz": ("float complex", "double complex"), "zc": ("double complex", "float complex")}


def database_path() -> str:
    """$TTC_ROOT/ttc/ttc.db like TTC when TTC_ROOT is set, else ~/.cache/ttc_b200/ttc.db."""
    if os.environ.get("TTC_B200_DB"):
        return os.environ["TTC_B200_DB"]
    if os.environ.get("TTC_ROOT"):
        d = Path(os.environ["TTC_ROOT"]) / "ttc"
    else:
        d = Path.home() / ".cache" / "ttc_b200"
    d.mkdir(parents=True, exist_ok=True)
    return str(d / "ttc.db")


def getTransposeName(ttcArgs) -> str:
    """TTC's name of the generated function for the cuda architecture (ttc.py:42-95), including its
    spelling "zs" for double complex -> float complex."""
    a, b = ttcArgs.floatTypeA, ttcArgs.floatTypeB
    if a == "float":
        name = "s" if b == "float" else "sd"
    elif a == "double":
        name = "d" if b == "double" else "ds"
    elif a == "float complex":
        name = "c" if b == "float complex" else "cz"
    else:
        name = "z" if b == "double complex" else "zs"
    name += "CuTranspose_" + "".join(str(p) for p in ttcArgs.idxPerm) + "_" + "x".join(str(s) for s in ttcArgs.size)
    if ttcArgs.beta == 0:
        name += "_bz"
    return name


def _function_name(ttcArgs) -> str:
    """Name of the emitted function (CUDAtranspose.py:473-527): the type prefix is derived from both
    types, e.g. "zc" for double complex -> float complex."""
    prefix = ttc_util.getFloatPrefix(ttcArgs.floatTypeA, ttcArgs.floatTypeB)
    name = prefix + "CuTranspose_" + "".join(str(p) for p in ttcArgs.idxPerm) + "_" + \
        "x".join(str(s) for s in ttcArgs.size)
    return name + ("_bz" if ttcArgs.beta == 0 else "")


def printEpilog(transposeName, ttcArgs):
    print(OKGREEN + "[SUCCESS]" + ENDC + " Please find the generated code under ./ttc_transpositions/%s.h\n"
          % transposeName)
    print("------------------ Usage ------------------")
    print("// 1) include header")
    print('#include "%s.h"' % transposeName)
    print("")
    print("// 2) execute transposition")
    if ttcArgs.beta != 0:
        print("%s(A, B, alpha, beta, size, lda, ldb);" % transposeName)
    else:
        print("%s(A, B, alpha, size, lda, ldb);" % transposeName)
    print("-------------------------------------------")


# ------------------------------------------------------------------------------------------------
CU_TYPE = {"float": "float", "double": "double", "float complex": "cuFloatComplex",
           "double complex": "cuDoubleComplex"}
SCALAR = {"float": "float", "double": "double", "float complex": "float", "double complex": "double"}
ENUM = {"float": "TTCB_S", "double": "TTCB_D", "float complex": "TTCB_C", "double complex": "TTCB_Z"}


def emit_shim(ttcArgs, file_name: str, func: str, tuning: dict, size, perm, lda, ldb) -> tuple[str, str]:
    """Header and source with TTC's exact entry point (CUDAtranspose.py:438-451) calling the C ABI."""
    ta, tb = ttcArgs.floatTypeA, ttcArgs.floatTypeB
    beta = ttcArgs.beta != 0
    sig = (f'extern "C" void {func}(const {CU_TYPE[ta]}* A, {CU_TYPE[tb]}* B, const {SCALAR[ta]} alpha'
           + (f", const {SCALAR[tb]} beta" if beta else "") + ", const int* size, const int* lda, const int* ldb)")
    guard = (file_name + "_H").upper()
    h = (f"#ifndef {guard}\n#define {guard}\n#include <cuComplex.h>\n{sig};\n")
    if file_name != func:
        alias = sig.replace(f" {func}(", f" {file_name}(")
        h += f"{alias};\n"
    h += "#endif\n"
    rank = len(size)
    from ._native import Tuning
    packed = Tuning.make(**tuning)  # an explicit loop order travels as raster_lo/raster_hi
    fields = " ".join(f"t.{k} = {int(getattr(packed, k))};" for k, _ in Tuning._fields_
                      if int(getattr(packed, k)) != 0)
    a_val = f"{SCALAR[ta]} a[2] = {{alpha, 0}};" if "complex" in ta else f"{SCALAR[ta]} a[1] = {{alpha}};"
    b_val = (f"{SCALAR[tb]} b[2] = {{beta, 0}};" if "complex" in tb else f"{SCALAR[tb]} b[1] = {{beta}};") \
        if beta else f"{SCALAR[tb]}* b = 0;"
    src = f"""// Generated by ttc_b200 for perm {perm}, size {size}, {ta} -> {tb}; tuned schedule {json.dumps(tuning)}.
#include <cuda_runtime.h>
#include <cuComplex.h>
#include <stdio.h>
#include <string.h>
#include "ttcb200.h"

{sig}
{{
  static ttcb_plan* plan = 0;
  static int64_t key[{3 * rank}];
  int64_t s[{rank}], la[{rank}], lb[{rank}], k[{3 * rank}];
  const int perm[{rank}] = {{{", ".join(map(str, perm))}}};
  for (int i = 0; i < {rank}; ++i) {{
    s[i] = size[i];
    la[i] = lda ? lda[i] : size[i];
    lb[i] = ldb ? ldb[i] : size[perm[i]];
    k[i] = s[i]; k[{rank} + i] = la[i]; k[{2 * rank} + i] = lb[i];
  }}
  if (!plan || memcmp(k, key, sizeof(key)) != 0) {{
    ttcb_tuning t;
    memset(&t, 0, sizeof(t));
    {fields}
    if (plan) ttcb_plan_destroy(plan);
    plan = 0;
    if (ttcb_plan_create(&plan, {rank}, perm, s, la, lb, {ENUM[ta]}, {ENUM[tb]}, {1 if beta else 0}, &t) != TTCB_OK) {{
      fprintf(stderr, "[TTC] ERROR in {func}: %s\\n", ttcb_last_error());
      return;
    }}
    memcpy(key, k, sizeof(key));
  }}
  {a_val}
  {b_val}
  if (ttcb_transpose(plan, A, B, a, b, 0) != TTCB_OK) fprintf(stderr, "[TTC] ERROR in {func}: %s\\n", ttcb_last_error());
  cudaError_t err = cudaDeviceSynchronize();
  if (err != cudaSuccess) fprintf(stderr, "[TTC] ERROR in {func}: %s\\n", cudaGetErrorString(err));
}}
"""
    if file_name != func:
        alias = sig.replace(f" {func}(", f" {file_name}(")
        call_b = ", beta" if beta else ""
        src += f"\n{alias}\n{{\n  {func}(A, B, alpha{call_b}, size, lda, ldb);\n}}\n"
    return h, src


# ------------------------------------------------------------------------------------------------
def _validate(a: TTCargs):
    if len(a.idxPerm) != len(a.size):
        raise TTCError(2, "dimension of permutation and size does not match.")
    if sorted(a.idxPerm) != list(range(len(a.idxPerm))):
        raise TTCError(3, "permutation is invalid.")
    if len(a.ldb) and len(a.ldb) != len(a.size):
        raise TTCError(4, "not all leading dimensions of B have been specified")
    if len(a.lda) and len(a.lda) != len(a.size):
        raise TTCError(4, "not all leading dimensions of A have been specified")
    for i, l in enumerate(a.ldb):
        if a.size[a.idxPerm[i]] > l:
            raise TTCError(4, "the leading dimension of B for dim %d is smaller than allowed (it must be >= %d)"
                           % (i, a.size[a.idxPerm[i]]))
    for i, l in enumerate(a.lda):
        if a.size[i] > l:
            raise TTCError(4, "the leading dimension of A for dim %d is smaller than allowed (it must be >= %d)"
                           % (i, a.size[i]))
    if (a.floatTypeA, a.floatTypeB) not in ttc_util.PREFIX:
        raise TTCError(5, "unknown precision. It needs to be either of the following s, d, c, z, sd, ds, cz, or zc.")


def _tunings_from_args(a: TTCargs, dtype: str):
    """Maps TTC's --blockings / --loopPerm / --threadsPerBlock restrictions onto schedule knobs."""
    from .autotune import knob_space
    space = knob_space(dtype)
    ea = ttc_util.getFloatTypeSize(a.floatTypeA)
    if a.blockings:
        space["tile_elems"] = sorted({int(bA) * int(bB) for bA, bB in a.blockings})
        space["run_bytes"] = sorted({int(bA) * ea for bA, _ in a.blockings})
    if a.loopPermutations:
        # each given loop order becomes the tile grid's raster, as given (no preset stands in)
        space["loop_order"] = []
        space["rasters"] = [list(lp) for lp in a.loopPermutations]
    else:
        # TTC ranks every loop order with its cost heuristic and keeps the cheapest
        space["rasters"] = ("ttc", 2)
    return space


def generateTransposition(ttcArgs: TTCargs):
    """Tunes (or looks up) the transposition described by ttcArgs, writes
    ./ttc_transpositions/<name>.{h,cu} and returns (transposeName, GiB/s of the fastest variant)."""
    from . import autotune
    from .core import plan_host_json

    a = ttcArgs
    if a.architecture != "cuda" and getattr(a, "architectureGiven", False):
        # a CPU architecture asked for explicitly: TTC's own CPU generator does the work
        from . import cpu_delegate
        if a.compiler == "nvcc":
            a.compiler = "g++"
        return cpu_delegate.generate(a, echo=not a.silent)
    if a.architecture != "cuda":
        if not a.silent:
            print(WARNING + "[TTC] WARNING: this implementation targets the GPU -> switching architecture to cuda "
                  "(--architecture=avx runs TTC's own CPU generator)." + ENDC)
        a.architecture = "cuda"
    a.compiler = "nvcc"
    if a.maxNumImplementations == -1:
        a.maxNumImplementations = 10000000
    a.lda = list(a.lda or [])
    a.ldb = list(a.ldb or [])
    _validate(a)
    for v in a.vecLength:
        if int(v) != 256 and not a.silent:
            print(WARNING + "[TTC] WARNING: the kernels use 256 threads per block; --threadsPerBlock=%d is ignored"
                  % int(v) + ENDC)

    # index fusion, reported like TTC (ttc.py:675-684)
    sizeOld, permOld, ldaOld, ldbOld = map(copy.deepcopy, (a.size, a.idxPerm, a.lda, a.ldb))
    fsize, fperm, flda, fldb = list(a.size), list(a.idxPerm), list(a.lda), list(a.ldb)
    ttc_util.fuseIndices(fsize, fperm, [], flda, fldb)
    flda, fldb = ttc_util.denseLeadingDims(fsize, fperm, flda, fldb)
    if len(fsize) != len(sizeOld) and not a.silent:
        print("Permutation and Size _before_ index-fusion: ", permOld, sizeOld, ldaOld, ldbOld)
        print("Permutation and Size _after_ index-fusion: ", fperm, fsize, flda, fldb)

    dtype = ttc_util.getFloatPrefix(a.floatTypeA, a.floatTypeB)
    alpha = complex(a.alpha) if "complex" in a.floatTypeA else float(a.alpha)
    beta = complex(a.beta) if "complex" in a.floatTypeB else float(a.beta)
    prob = autotune.Problem(list(a.idxPerm), list(a.size), dtype, alpha, beta, a.lda or None, a.ldb or None)
    arch = ttc_util.getArchitecture("cuda")
    db = getattr(a, "database", None) or database_path()
    transposeName = getTransposeName(a)
    func = _function_name(a)

    if not a.silent:
        print("--------------Settings---------------------")
        print("Device: ".ljust(20) + arch.strip())
        print("Beta:".ljust(20) + "%f" % a.beta)
        version = ttc_util.getVersion()
        print("Version:".ljust(20) + "v%d.%d.%d" % (version[0], version[1], version[2]))
        print("-------------------------------------------")

    best_tuning, best_gibps, variants, measuring = None, 0.0, [], 0.0
    if not a.ignoreDatabase:
        try:
            hit = sql_util.lookup(db, fsize, fperm, a.floatTypeA, a.floatTypeB, a.beta, arch)
        except sql_util.DatabaseUnavailable as e:
            hit = None
            if not a.silent:
                print(WARNING + f"[TTC] WARNING: {e}; falling back to a measured search" + ENDC)
        if hit is not None:
            best_tuning, best_gibps = hit["tuning"], hit["bandwidth"]
            if not a.silent:
                print("Solution already exists: generating the solution which was found previously.")

    if best_tuning is None:
        if a.generateOnly:
            best_tuning = {}
        else:
            t0 = time.perf_counter()
            if getattr(a, "model", 0):
                from . import cost_model
                sel = cost_model.select(prob, max_impl=a.maxNumImplementations,
                                        confidence=a.confidence or None, verify=not a.noTest)
                results = sel["results"]
            else:
                space = _tunings_from_args(a, dtype)
                cands = autotune.candidate_tunings(prob, a.maxNumImplementations, space)
                if not a.silent:
                    print("[running] measure runtime of %d schedules" % len(cands))
                results = autotune.measure(prob, cands, reps=4, verify=not a.noTest)
            measuring = time.perf_counter() - t0
            bad = [r for r in results if not r.ok]
            if bad:
                raise TTCError(1, "[TTC_Error] %d out of %d tests failed." % (len(bad), len(results)))
            if not a.silent:
                print(OKGREEN + "[Success] all %d tests passed." % len(results), ENDC)
            order = sorted(results, key=lambda r: r.time_ms)
            best = order[0]
            best_tuning = best.tuning
            best_gibps = prob.bytes() / (best.time_ms * 1e-3) / (1 << 30)
            for rank, r in enumerate(order):
                t = r.desc.get("tile") or {}
                variants.append({"tuning": r.tuning, "bandwidth": prob.bytes() / (r.time_ms * 1e-3) / (1 << 30),
                                 "time": r.time_ms * 1e-3, "rank": rank, "blockA": t.get("LA", 0),
                                 "blockB": t.get("LB", 0)})
            if not a.silent:
                print("Measuring took %f seconds" % measuring)
                print("\nThe fastest version (%s) attains %.2f GiB/s.\n" % (json.dumps(best_tuning), best_gibps))

    # emit the winner (ttc.py:1027-1070)
    out_dir = Path.cwd() / "ttc_transpositions"
    out_dir.mkdir(exist_ok=True)
    h, src = emit_shim(a, transposeName, func, best_tuning, list(a.size), list(a.idxPerm), a.lda or None,
                       a.ldb or None)
    (out_dir / f"{transposeName}.h").write_text(h)
    (out_dir / f"{transposeName}.cu").write_text(src)
    (out_dir / f"{transposeName}.json").write_text(json.dumps(
        {"perm": a.idxPerm, "size": a.size, "dtype": dtype, "lda": a.lda, "ldb": a.ldb, "beta_nonzero": a.beta != 0,
         "tuning": best_tuning, "plan": plan_host_json(prob.perm, prob.size, dtype, prob.beta_nonzero, prob.lda,
                                                       prob.ldb, best_tuning or None)}, indent=1))

    if variants and a.updateDatabase:
        try:
            sql_util.insert(db, fsize, fperm, a.floatTypeA, a.floatTypeB, a.alpha, a.beta, arch,
                            socket.gethostname(), variants, measuring)
        except sql_util.DatabaseUnavailable as e:
            if not a.silent:
                print(WARNING + f"[TTC] WARNING: results not stored: {e}" + ENDC)
    if not a.silent:
        printEpilog(transposeName, a)
    return (transposeName, best_gibps)


def load_transposition(name: str, directory: str | Path = "ttc_transpositions"):
    """A callable `transpose(A, B, alpha, beta)` for a generated transposition (torch CUDA tensors)."""
    from .core import Plan
    meta = json.loads((Path(directory) / f"{name}.json").read_text())
    plan = Plan(meta["perm"], meta["size"], meta["dtype"], meta["beta_nonzero"], meta["lda"] or None,
                meta["ldb"] or None, meta["tuning"] or None)

    def transpose(A, B, alpha=1.0, beta=0.0, stream=None):
        plan(A, B, alpha, beta, stream)

    transpose.plan = plan
    return transpose


# ------------------------------------------------------------------------------------------------
def parse_args(argv) -> TTCargs:
    """TTC's argument parsing (ttc.py:1132-1338), same flags and defaults."""
    o = {"perm": [], "size": [], "lda": [], "ldb": [], "alpha": 1.0, "beta": 0.0, "maxImpl": 200,
         "floatA": "float", "floatB": "float", "arch": "avx", "compiler": "icpc", "blockings": [], "loopPerms": [],
         "vec": [], "flags": set(), "numThreads": 0, "affinity": "", "prefetch": [], "model": 0, "confidence": 0.0,
         "database": None}
    for arg in argv:
        key = arg.split("=")[0]
        if key not in ALLOWED:
            raise TTCError(1, "Error: argument " + key + " not valid.")
        val = arg.split("=", 1)[1] if "=" in arg else None
        if val is None:
            o["flags"].add(key)
            continue
        if key == "--architecture":
            if val not in ("avx", "knc", "avx512", "power", "cuda"):
                raise TTCError(1, "[TTC] ERROR: Architecture unknown.")
            o["arch"] = val
            o["arch_given"] = True
        elif key == "--compiler":
            if val not in ("icpc", "g++", "ibm", "nvcc"):
                raise TTCError(1, "[TTC] ERROR: unknown compiler choice.")
            o["compiler"] = val
            if val == "nvcc":
                o["arch"] = "cuda"
        elif key in ("--dataType", "--floatType"):
            if val not in DTYPE_ARG:
                raise TTCError(5, "[TTC] ERROR: unknown precision. It needs to be either of the following s, d, c, "
                                  "z, sd, ds, cz, or zc.")
            o["floatA"], o["floatB"] = DTYPE_ARG[val]
        elif key == "--alpha":
            o["alpha"] = float(val)
        elif key == "--beta":
            o["beta"] = float(val)
        elif key == "--maxImplementations":
            o["maxImpl"] = int(val)
        elif key == "--numThreads":
            o["numThreads"] = int(val)
        elif key == "--affinity":
            o["affinity"] = val
        elif key == "--prefetchDistances":
            o["prefetch"] = [int(x) for x in val.split(",")]
        elif key == "--blockings":
            o["blockings"] = [(int(b.split("x")[0]), int(b.split("x")[1])) for b in val.split(",")]
        elif key == "--threadsPerBlock":
            for v in val.split(","):
                if int(v) not in (128, 256, 512):
                    raise TTCError(1, "[TTC] ERROR: value for --threadsPerBlock is not valid. It needs to be either "
                                      "128, 256 or 512.")
                o["vec"].append(int(v))
        elif key == "--size":
            o["size"] = [int(s) for s in val.split(",")]
        elif key == "--perm":
            o["perm"] = [int(s) for s in val.split(",")]
        elif key == "--lda":
            o["lda"] = [int(s) for s in val.split(",")]
        elif key == "--ldb":
            o["ldb"] = [int(s) for s in val.split(",")]
        elif key == "--loopPerm":
            o["loopPerms"] = [[int(x) for x in lp.split(",")] for lp in val.split("-")]
        elif key == "--model":
            o["model"] = int(val)
        elif key == "--confidence":
            o["confidence"] = float(val)
        elif key == "--database":
            o["database"] = val
    if len(o["perm"]) != len(o["size"]):
        raise TTCError(2, "[Error] dimension of permutation and size does not match.")
    a = TTCargs(o["perm"], o["size"])
    a.alpha, a.beta = o["alpha"], o["beta"]
    a.maxNumImplementations = o["maxImpl"]
    a.floatTypeA, a.floatTypeB = o["floatA"], o["floatB"]
    a.architecture, a.compiler = o["arch"], o["compiler"]
    a.architectureGiven = bool(o.get("arch_given"))
    a.lda, a.ldb = o["lda"], o["ldb"]
    a.blockings, a.loopPermutations, a.vecLength = o["blockings"], o["loopPerms"], o["vec"]
    a.numThreads, a.affinity, a.prefetchDistances = o["numThreads"], o["affinity"], o["prefetch"]
    f = o["flags"]
    a.keep = int("--keep" in f)
    a.ignoreDatabase = int("--ignoreDatabase" in f)
    a.generateOnly = int("--generateOnly" in f)
    a.noTest = int("--noTest" in f)
    a.streamingStores = int("--streamingStores" in f or "--use-streamingStores" in f)
    a.align = 0 if "--no-align" in f else 1
    a.scalar = int("--no-vec" in f)
    a.debug = int("-v" in f or "--verbose" in f)
    a.hotA, a.hotB = int("--hotA" in f), int("--hotB" in f)
    a.batched = int("--batched" in f)
    if "--model" in f:
        a.model = 1
    else:
        a.model = o["model"]
    a.confidence = o["confidence"]
    a.database = o["database"]
    a.showHelp = "--help" in f
    return a


def printHelp():
    print("Usage: ttc --perm=..., --size=... [optional arguments]\n")
    print("   B_{Pi(i1,i2,..., iN)} = alpha * A_{i1,i2,..., iN} + beta * B_{Pi(i1,i2,..., iN)}\n")
    print("required arguments:")
    print("   --perm=<index1>,<index2>,...,<indexN>".ljust(60), "specify the permutation")
    print("   --size=<size1>,<size2>,...,<sizeN>".ljust(60), "size of the input tensor")
    print("optional arguments (as in TTC): --lda --ldb --maxImplementations --alpha --beta --dataType")
    print("   --blockings --loopPerm --threadsPerBlock --generateOnly --noTest --keep --ignoreDatabase")
    print("additions: --model (learned schedule selection), --confidence=<0..1>, --database=<path>")
    print("\nExample: \"ttc --perm=1,0,2 --size=1000,768,16 --beta=1.0 --dataType=s --architecture=cuda\"")


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    try:
        a = parse_args(argv)
        if not argv or a.showHelp:
            printHelp()
            return 0
        generateTransposition(a)
        return 0
    except TTCError as e:
        printHelp()
        print(FAIL + str(e) + ENDC)
        return 1


if __name__ == "__main__":
    sys.exit(main())
