"""TTC's own CUDA kernels on the B200, beside this library's.

When oracle/_ref/libttc_ref_cuda.so is present (TTC's CUDA generator, run by oracle/make_ref_gpu.py
where the TTC sources are, compiled for sm_100a), its first variant for a sample of the 64-case sweep
runs through TTC's own generated wrapper on the benchmark's inputs. Its results must agree with the
oracle and with this library: bit for bit when beta = 0 (both compute alpha*A in A's precision), and
within one unit in the last place of the larger term when beta != 0 (nvcc may contract TTC's
alpha*A + beta*B into a fused multiply-add, CUDAtranspose.py:801-900 in the TTC project; this library
rounds both products).
"""
import math
import os

import numpy as np
import pytest

import oracle
from oracle import cuda_ref

pytestmark = pytest.mark.gpu

SAMPLE = [0, 1, 6, 7, 11, 24, 40, 41]


@pytest.mark.skipif(cuda_ref.available() is None, reason="TTC's CUDA kernels were not built (needs the TTC sources)")
@pytest.mark.parametrize("case", SAMPLE)
def test_ttc_cuda_kernels_agree_with_oracle_and_library(case):
    import torch
    import ttc_b200.workloads as wl
    from ttc_b200 import Plan
    from helpers import assert_bitexact
    ref = cuda_ref.available()
    c = wl.sweep_cases(2024)[case]
    if not ref.covers(c):
        pytest.skip("case not built")
    tmap = {"s": torch.float32, "d": torch.float64}
    n = math.prod(c["size"])
    gen = torch.Generator(device="cuda")
    gen.manual_seed(c["seed"])
    A = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen).mul_(2).sub_(1)
    gen.manual_seed(c["seed"] + 1)
    B0 = torch.rand(n, dtype=tmap[c["dtype"]], device="cuda", generator=gen).mul_(2).sub_(1)
    B_ttc, B_ours = B0.clone(), B0.clone()
    ref.call(c, 0, A.data_ptr(), B_ttc.data_ptr())
    plan = Plan(c["perm"], c["size"], c["dtype"], c["beta"] != 0)
    plan(A, B_ours, c["alpha"], c["beta"])
    torch.cuda.synchronize()
    want = B0.cpu().numpy().copy()
    oracle.transpose(A.cpu().numpy(), want, c["perm"], c["size"], c["alpha"], c["beta"], dtype=c["dtype"],
                     threads=os.cpu_count() or 1)
    got_ttc, got_ours = B_ttc.cpu().numpy(), B_ours.cpu().numpy()
    assert_bitexact(got_ours, want, f"library, case {case}")
    if c["beta"] == 0:
        assert_bitexact(got_ttc, want, f"TTC's CUDA kernel, case {case}")
    else:
        # a fused multiply-add skips the rounding of one product: the results differ by at most one
        # unit in the last place of the larger term (not of the result, which cancellation can make
        # tiny), as for TTC's CPU code (tests/test_reference_cpu.py)
        real = np.float32 if c["dtype"] == "s" else np.float64
        t = oracle.transpose(A.cpu().numpy(), np.zeros_like(want), c["perm"], c["size"], c["alpha"], 0.0,
                             dtype=c["dtype"], threads=os.cpu_count() or 1)
        scale = np.maximum(np.abs(t), np.abs(real(c["beta"]) * B0.cpu().numpy()))
        tol = np.spacing(scale.astype(real)) + np.spacing(np.abs(want))
        assert np.all(np.abs(got_ttc.astype(np.float64) - want.astype(np.float64)) <= tol), f"TTC, case {case}"
    plan.close()
