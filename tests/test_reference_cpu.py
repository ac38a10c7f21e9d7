"""When oracle/_ref (TTC's own generated AVX code for the sweep cases, built by oracle/make_ref.py
where the TTC sources are available) is present, its outputs must equal the oracle's. This checks the
oracle against the reference implementation itself at full size, on the host, on a sample of the
64 cases spread over ranks, types and both alpha/beta settings."""
import math

import numpy as np
import pytest

import oracle
from oracle import cpu_ref


@pytest.mark.skipif(cpu_ref.available() is None, reason="oracle/_ref was not built (needs the TTC sources)")
@pytest.mark.parametrize("case", [0, 1, 2, 3, 11, 24, 40, 41, 57, 63])
def test_ttc_generated_cpu_code_matches_oracle(case):
    import ttc_b200.workloads as wl
    run = cpu_ref.available()
    c = wl.sweep_cases(2024)[case]
    if cpu_ref._key(c) not in run.keys:
        pytest.skip("case not in the built sample")
    real = np.float32 if c["dtype"] == "s" else np.float64
    n = math.prod(c["size"])
    A = cpu_ref.aligned(n, real)
    B = cpu_ref.aligned(n, real)
    A[:] = np.random.default_rng(c["seed"]).uniform(-1, 1, n)
    B[:] = np.random.default_rng(c["seed"] + 1).uniform(-1, 1, n)
    Bc = cpu_ref.aligned(n, real)
    Bc[:] = B
    got = run(c, A, Bc, 4)
    want = oracle.transpose(A, B.copy(), c["perm"], c["size"], c["alpha"], c["beta"], dtype=c["dtype"], threads=4)
    if c["beta"] == 0:
        assert np.array_equal(got, want)
    else:
        # TTC's AVX code fuses beta*B + (alpha*A) into one FMA (transposeGenerator.py:1048-1049), which
        # skips one rounding of beta*B. The two results then differ by at most one unit in the last
        # place of the larger operand (not of the result, which cancellation can make tiny).
        t = oracle.transpose(A, np.zeros_like(B), c["perm"], c["size"], c["alpha"], 0.0, dtype=c["dtype"],
                             threads=4)
        scale = np.maximum(np.abs(t), np.abs(real(c["beta"]) * B))
        tol = np.spacing(scale.astype(real)) + np.spacing(np.abs(want))
        assert np.all(np.abs(got.astype(np.float64) - want.astype(np.float64)) <= tol)
