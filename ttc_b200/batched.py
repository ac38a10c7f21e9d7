"""Batched mode: many independent transpositions in one persistent kernel launch, optionally replayed
from a captured CUDA graph. Each problem keeps the schedule of its own plan (which the autotuner or
the learned selector chose)."""
from __future__ import annotations

import ctypes
from typing import Sequence

from ._native import TTCError, check, lib
from .core import Plan, _ptr, _stream_handle, pack_scalar


class Batch:
    """``Batch(plans, As, Bs, alpha, beta)`` binds device buffers to plans (same dtype pair and beta
    flag for all). ``launch()`` runs every problem in one launch; ``launch(graph=True)`` captures the
    launch (counter reset + kernel) into a CUDA graph once and replays it."""

    def __init__(self, plans: Sequence[Plan], As, Bs, alpha=1.0, beta=0.0, blocks: int = 0):
        if not plans:
            raise TTCError(1, "empty batch")
        if len(plans) != len(As) or len(plans) != len(Bs):
            raise TTCError(1, "plans, As and Bs must have the same length")
        p0 = plans[0]
        self.plans = list(plans)  # keep the plans (and their tensors) alive with the batch
        self._keep = (list(As), list(Bs))
        n = len(plans)
        hp = (ctypes.c_void_p * n)(*[p.handle for p in plans])
        ha = (ctypes.c_void_p * n)(*[_ptr(a) for a in As])
        hb = (ctypes.c_void_p * n)(*[_ptr(b) for b in Bs])
        al = pack_scalar(p0.ta, alpha)
        be = pack_scalar(p0.tb, beta) if p0.beta_nonzero else None
        self._h = ctypes.c_void_p()
        check(lib().ttcb_batch_create(ctypes.byref(self._h), n, hp, ha, hb, ctypes.cast(al, ctypes.c_void_p),
                                      ctypes.cast(be, ctypes.c_void_p) if be is not None else None, int(blocks)))

    @property
    def bytes(self) -> int:
        return int(lib().ttcb_batch_bytes(self._h))

    def launch(self, stream=None, graph: bool = False) -> None:
        s = _stream_handle(stream)
        if graph:
            check(lib().ttcb_batch_graph_launch(self._h, s))
        else:
            check(lib().ttcb_batch_launch(self._h, s))

    def check_status(self, stream=None) -> None:
        """Reads the device status word of the last launch (synchronizes the stream)."""
        check(lib().ttcb_batch_status(self._h, _stream_handle(stream)))

    def close(self) -> None:
        if self._h.value:
            lib().ttcb_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
