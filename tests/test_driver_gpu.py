"""TTC's driver end to end on the GPU: generateTransposition tunes, stores and emits; a second call
hits the database; the emitted shim, compiled and linked into a C program, computes the oracle's
result through TTC's exact entry point; the measured search and the learned path agree."""
import json
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from helpers import assert_bitexact, make_inputs

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture
def workdir(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    monkeypatch.setenv("TTC_B200_DB", str(tmp_path / "ttc.db"))
    return tmp_path


def test_generate_transposition_and_database_hit(workdir, capsys):
    import torch
    from ttc_b200 import ttc, ttc_util
    a = ttc_util.TTCargs([1, 0, 2], [300, 257, 5])
    a.architecture = "cuda"
    a.beta = 1.0
    a.maxNumImplementations = 12
    a.silent = 1
    name, gibps = ttc.generateTransposition(a)
    assert name == "sCuTranspose_102_300x257x5" and gibps > 0
    assert (workdir / "ttc_transpositions" / f"{name}.h").exists()
    # second call: the database has it
    a2 = ttc_util.TTCargs([1, 0, 2], [300, 257, 5])
    a2.architecture = "cuda"
    a2.beta = 1.0
    name2, gibps2 = ttc.generateTransposition(a2)
    assert name2 == name and abs(gibps2 - gibps) < 1e-6
    assert "Solution already exists" in capsys.readouterr().out
    # the Python handle computes the oracle's result
    tr = ttc.load_transposition(name, workdir / "ttc_transpositions")
    A, B = make_inputs([300, 257, 5], [1, 0, 2], "s", 3)
    want = oracle.transpose(A, B.copy(), [1, 0, 2], [300, 257, 5], 1.0, 1.0)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    tr(dA, dB, 1.0, 1.0)
    torch.cuda.synchronize()
    assert_bitexact(dB.cpu().numpy(), want, "load_transposition")


def test_cli_main(workdir):
    from ttc_b200 import ttc
    rc = ttc.main(["--perm=2,0,1", "--size=33,17,9", "--dataType=zc", "--alpha=0.5", "--architecture=cuda",
                   "--maxImplementations=6", "--ignoreDatabase"])
    assert rc == 0
    assert (workdir / "ttc_transpositions" / "zsCuTranspose_201_33x17x9_bz.h").exists()


@pytest.mark.parametrize("dtype,beta", [("s", 1.0), ("zc", 0.0), ("ds", -0.5)])
def test_generated_shim_links_and_matches_oracle(workdir, dtype, beta):
    """The emitted extern "C" function, with TTC's name and signature, linked into a host program."""
    from ttc_b200 import ttc, ttc_util
    perm, size, lda = [2, 0, 1], [13, 9, 6], [16, 9, 6]
    a = ttc_util.TTCargs(perm, size)
    a.floatTypeA, a.floatTypeB = ttc_util.TYPES_OF_PREFIX[dtype]
    a.architecture, a.beta, a.alpha, a.lda, a.silent = "cuda", beta, 1.5, list(lda), 1
    a.maxNumImplementations = 4
    a.ignoreDatabase = 1
    name, _ = ttc.generateTransposition(a)
    func = ttc._function_name(a)
    A, B = make_inputs(size, perm, dtype, 9, lda)
    want = oracle.transpose(A, B.copy(), perm, size, 1.5, beta, lda, None, dtype)
    ta, tb = ttc_util.TYPES_OF_PREFIX[dtype]
    cu = {"float": "float", "double": "double", "float complex": "cuFloatComplex", "double complex": "cuDoubleComplex"}
    sc = {"float": "float", "double": "double", "float complex": "float", "double complex": "double"}
    beta_arg = f", ({sc[tb]}){beta}" if beta != 0 else ""
    prog = f"""
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#include "{name}.h"
int main(int argc, char** argv) {{
  size_t na = {A.size}, nb = {B.size};
  FILE* f = fopen(argv[1], "rb");
  {cu[ta]}* hA = ({cu[ta]}*)malloc(na * sizeof({cu[ta]}));
  {cu[tb]}* hB = ({cu[tb]}*)malloc(nb * sizeof({cu[tb]}));
  if (fread(hA, sizeof({cu[ta]}), na, f) != na || fread(hB, sizeof({cu[tb]}), nb, f) != nb) return 2;
  fclose(f);
  {cu[ta]}* dA; {cu[tb]}* dB;
  cudaMalloc(&dA, na * sizeof({cu[ta]})); cudaMalloc(&dB, nb * sizeof({cu[tb]}));
  cudaMemcpy(dA, hA, na * sizeof({cu[ta]}), cudaMemcpyHostToDevice);
  cudaMemcpy(dB, hB, nb * sizeof({cu[tb]}), cudaMemcpyHostToDevice);
  int size[] = {{{", ".join(map(str, size))}}}, lda[] = {{{", ".join(map(str, lda))}}}, ldb[] = {{{", ".join(str(size[p]) for p in perm)}}};
  {func}(dA, dB, ({sc[ta]})1.5{beta_arg}, size, lda, ldb);
  cudaMemcpy(hB, dB, nb * sizeof({cu[tb]}), cudaMemcpyDeviceToHost);
  f = fopen(argv[2], "wb"); fwrite(hB, sizeof({cu[tb]}), nb, f); fclose(f);
  return 0;
}}
"""
    (workdir / "prog.cu").write_text(prog)
    (workdir / "in.bin").write_bytes(A.tobytes() + B.tobytes())
    lib_dir = ROOT / "ttc_b200"
    cmd = ["/usr/local/cuda/bin/nvcc", "-o", str(workdir / "prog"), str(workdir / "prog.cu"),
           str(workdir / "ttc_transpositions" / f"{name}.cu"), "-I", str(workdir / "ttc_transpositions"),
           "-I", str(ROOT / "include"), str(lib_dir / "libttcb200.so"), f"-Xlinker=-rpath={lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(workdir / "prog"), str(workdir / "in.bin"), str(workdir / "out.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    got = np.frombuffer((workdir / "out.bin").read_bytes(), dtype=want.dtype)
    assert_bitexact(got, want, f"shim {name}")


def test_measured_search_verifies_and_ranks():
    from ttc_b200.autotune import Problem, candidate_tunings, search
    p = Problem([2, 0, 1], [7, 3, 200001], "s", 1.5, -0.5)
    r = search(p, max_impl=16, reps=3)
    distinct = len(candidate_tunings(p, 1000))
    assert r["candidates"] == min(16, distinct) >= 8 and all(x.ok for x in r["results"])
    assert r["best"].gbs == max(x.gbs for x in r["results"])
