"""ttc_b200 - B200-native out-of-place tensor transposition with TTC's interface.

    B_{perm(i0..iN-1)} = alpha * A_{i0..iN-1} + beta * B_{perm(i0..iN-1)}

Python host side over the C ABI of ``libttcb200.so`` (include/ttcb200.h), whose kernels are
hand-written for sm_100a. There is no CPU fallback: the first call that needs the library loads it
and raises ImportError if it is missing (``python -m ttc_b200.build`` builds it in-tree).
"""
from ._native import TTCError, Tuning
from .core import Plan, transpose, plan_host_json, fuse, VALID_DTYPES, FLOAT_TYPES

__all__ = ["Plan", "transpose", "TTCError", "Tuning", "plan_host_json", "fuse", "VALID_DTYPES", "FLOAT_TYPES"]
__version__ = "0.1.0"
