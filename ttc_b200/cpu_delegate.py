"""CPU architectures through the same command line: `--architecture=avx|avx512|knc|power`.

TTC generates C++ for CPUs (transposeGenerator.py, transpose.py) and CUDA for GPUs from one driver
(ttc.py:614-1130, CLI :1132-1376). This library replaces the CUDA path; a request for a CPU
architecture is handed, with the same flags, to TTC's own driver run from a TTC checkout (the
directory in $TTC_SOURCE_DIR), converted to Python 3 by ttc_b200.py2compat. TTC then generates,
compiles, measures and writes ttc_transpositions/<name>.h in the current directory exactly as it
would on its own. Without a TTC checkout the request fails with a message saying so; it never falls
back to the GPU or to anything else.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile
from pathlib import Path

from ._native import TTCError
from . import ttc_util

CPU_ARCHITECTURES = ("avx", "avx512", "knc", "power")
PACKAGE = ["ttc", "ttc_util", "sql_util", "transpose", "transposeGenerator", "GPUtransposeGenerator",
           "CUDAtranspose", "GPUreference"]


def source_dir() -> Path:
    d = os.environ.get("TTC_SOURCE_DIR", "")
    if not d or not (Path(d) / "ttc" / "ttc.py").exists():
        raise TTCError(9, "[TTC] ERROR: --architecture=avx|avx512|knc|power runs TTC's own CPU code generator, "
                          "which needs the TTC sources: set TTC_SOURCE_DIR to a TTC checkout")
    return Path(d)


def to_argv(a) -> list[str]:
    """TTC's command line for a TTCargs (ttc.py:1132-1338)."""
    prefix = ttc_util.getFloatPrefix(a.floatTypeA, a.floatTypeB)
    argv = [f"--perm={','.join(map(str, a.idxPerm))}", f"--size={','.join(map(str, a.size))}",
            f"--dataType={prefix}", f"--alpha={a.alpha}", f"--beta={a.beta}",
            f"--architecture={a.architecture}", f"--compiler={a.compiler}",
            f"--maxImplementations={a.maxNumImplementations}"]
    if a.lda:
        argv.append(f"--lda={','.join(map(str, a.lda))}")
    if a.ldb:
        argv.append(f"--ldb={','.join(map(str, a.ldb))}")
    if a.numThreads:
        argv.append(f"--numThreads={a.numThreads}")
    if a.affinity:
        argv.append(f"--affinity={a.affinity}")
    if a.blockings:
        argv.append("--blockings=" + ",".join(f"{x}x{y}" for x, y in a.blockings))
    if a.loopPermutations:
        argv.append("--loopPerm=" + "-".join(",".join(map(str, lp)) for lp in a.loopPermutations))
    if a.prefetchDistances:
        argv.append("--prefetchDistances=" + ",".join(map(str, a.prefetchDistances)))
    for flag, on in (("--keep", a.keep), ("--ignoreDatabase", a.ignoreDatabase), ("--noTest", a.noTest),
                     ("--no-align", not a.align), ("--no-vec", a.scalar), ("--hotA", a.hotA), ("--hotB", a.hotB),
                     ("--streamingStores", a.streamingStores)):
        if on:
            argv.append(flag)
    return argv


def generate(a, cwd: str | None = None, echo: bool = True) -> tuple[str, float]:
    """Runs TTC's driver for a CPU architecture; returns (transposition name, GiB/s of the fastest
    variant) as TTC reports them. The generated header lands in <cwd>/ttc_transpositions."""
    src = source_dir()
    from .py2compat import convert_tree
    work = Path(tempfile.mkdtemp(prefix="ttc_cpu_"))
    convert_tree(src / "ttc", work / "ttc", PACKAGE)
    (work / "ttc" / "__init__.py").write_text("from . import ttc\n")
    env = dict(os.environ, TTC_ROOT=str(work))
    code = ("import sys; sys.path.insert(0, %r); sys.argv = ['ttc'] + %r; from ttc.ttc import main; main()"
            % (str(work), to_argv(a)))
    cwd = cwd or os.getcwd()
    before = set((Path(cwd) / "ttc_transpositions").glob("*.h"))
    r = subprocess.run([sys.executable, "-c", code], cwd=cwd, env=env, capture_output=True, text=True)
    if echo:
        sys.stdout.write(r.stdout)
    m = re.search(r"fastest version \(([^)]*)\) attains ([0-9.]+) GiB/s", r.stdout)
    new = sorted(set((Path(cwd) / "ttc_transpositions").glob("*.h")) - before)
    if r.returncode != 0 or not m:
        raise TTCError(1, "[TTC] ERROR: TTC's CPU generator failed: " + (r.stdout + r.stderr)[-1500:])
    name = next((h.stem for h in new if h.name != "ttc_offset.h"), m.group(1))
    return name, float(m.group(2))
