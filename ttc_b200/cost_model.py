"""Learned schedule selection: an MLP that ranks the autotuner's candidate schedules.

TTC picks a transposition's variant by compiling and timing every candidate (ttc.py:847-1022,
GPUtransposeGenerator.py:165-230). Here a 3-layer fp32 MLP (128 hidden units) predicts log(GB/s)
of every candidate schedule from problem and schedule features; the top prediction is used directly
when the model is confident, otherwise the top-k predictions are measured (a short measured search).

Features: rank, the permutation as one-hot, log2 extents, log2 strides of A and B, element sizes,
beta != 0, and the candidate's tile (size, run lengths), access widths, tile kernel variant, grid
raster order and CTA count (with the grid's waves and the strides between consecutive tiles), plus
the planner's own cost estimate. Candidates are described by shape-only plans (no descriptor
tables), so featurising a problem's candidates costs one host call.

The network is trained on the GPU with the library's own kernels (include/ttcb200_mlp.h: tiled GEMM
with fused bias/ReLU, ReLU backward, column sums, MSE, Adam) on timings the measured search itself
produced (`collect`). `python -m ttc_b200.cost_model collect|train|evaluate ...` runs each step.
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import math
import time
from pathlib import Path
from typing import Optional

import numpy as np

from . import _native
from .autotune import Problem, candidate_tunings, measure, Bench, staged_claims
from .core import ELEM_BYTES, plan_shapes, split_dtype

MAXD = 6
DEFAULT_MODEL = Path(__file__).resolve().parent / "data" / "cost_model.npz"
VERSION = "ttcb-mlp-v4"


# ------------------------------------------------------------------------------------------------
def problem_features(p: Problem, desc: dict) -> list[float]:
    r = len(p.size)
    f = [r / MAXD]
    onehot = [0.0] * (MAXD * MAXD)
    for j, d in enumerate(p.perm[:MAXD]):
        if d < MAXD:
            onehot[j * MAXD + d] = 1.0
    f += onehot
    ext = [math.log2(max(s, 1)) / 20.0 for s in p.size[:MAXD]]
    f += ext + [0.0] * (MAXD - len(ext))
    la = p.lda or p.size
    lb = p.ldb or [p.size[q] for q in p.perm]
    sA = [1] * r
    sBp = [1] * r
    for i in range(1, r):
        sA[i] = sA[i - 1] * la[i - 1]
        sBp[i] = sBp[i - 1] * lb[i - 1]
    sB = [0] * r
    for j, q in enumerate(p.perm):
        sB[q] = sBp[j]
    ls = [math.log2(max(x, 1)) / 30.0 for x in sA[:MAXD]]
    f += ls + [0.0] * (MAXD - len(ls))
    ls = [math.log2(max(x, 1)) / 30.0 for x in sB[:MAXD]]
    f += ls + [0.0] * (MAXD - len(ls))
    ta, tb = split_dtype(p.dtype)
    f += [ELEM_BYTES[ta] / 16.0, ELEM_BYTES[tb] / 16.0, 1.0 if p.beta_nonzero else 0.0,
          math.log2(max(p.elements(), 1)) / 30.0]
    fu = desc["fused"]
    f += [fu["rank"] / MAXD, 1.0 if fu["perm"] and fu["perm"][0] == 0 else 0.0]
    return f


def _shape_part(p: Problem, desc: dict) -> tuple:
    """The features of a candidate that depend only on its plan (tile shape), not on the launch
    knobs: (static values, tile count, tile bytes)."""
    ta, tb = split_dtype(p.dtype)
    t = desc.get("tile") or {}
    row = desc.get("row") or {}
    is_tile = desc["kernel"] == "tile"
    P = t.get("P", row.get("chunk", 1))
    LA = t.get("LA", row.get("w", 1))
    LB = t.get("LB", row.get("w", 1))
    nt = t.get("ntiles", row.get("units", 1))
    head = [1.0 if is_tile else 0.0, 0.0 if is_tile else 1.0,
            math.log2(max(P, 1)) / 14.0, math.log2(max(LA, 1)) / 14.0, math.log2(max(LB, 1)) / 14.0,
            desc["vecA"] / 4.0, desc["vecB"] / 4.0,
            math.log2(max(LA * ELEM_BYTES[ta], 1)) / 16.0, math.log2(max(LB * ELEM_BYTES[tb], 1)) / 16.0]
    mid = [min(desc["est_cost"], 200.0) / 32.0, math.log2(max(nt, 1)) / 25.0, float(t.get("fast", 0))]
    tail = [math.log2(max(P * ELEM_BYTES[ta], 1)) / 16.0,
            math.log2(max(P / max(LA, 1), 1)) / 10.0, math.log2(max(P / max(LB, 1), 1)) / 10.0]
    tile_bytes = P * (ELEM_BYTES[ta] + ELEM_BYTES[tb] * (2 if p.beta_nonzero else 1))
    return head, mid, tail, nt, tile_bytes


def _raster_jumps(p: Problem, tuning: dict, desc: dict, groups) -> list[float]:
    """The raster the candidate runs: whether it is the planner's choice, a preset or an explicit
    loop order, and the strides (log2 bytes, in A and in B) between consecutive tiles along its
    fastest and its second grid dimension."""
    from .autotune import grid_raster, preset_order
    ta, tb = split_dtype(p.dtype)
    fu = desc["fused"]
    t = desc.get("tile") or {}
    ext = t.get("ext") or [0] * fu["rank"]
    if tuning.get("raster") and groups is not None:
        order = []
        for d in tuning["raster"]:
            fd = next((i for i, g in enumerate(groups) if d in g), None)
            if fd is not None and fd not in order:
                order.append(fd)
        kind = [0.0, 0.0, 1.0]
    else:
        order = preset_order(desc, tuning.get("loop_order", 0))
        kind = [1.0 if not tuning.get("loop_order") else 0.0, 1.0 if tuning.get("loop_order") else 0.0, 0.0]
    grid = list(grid_raster(desc, order)) if desc["kernel"] == "tile" else []
    out = []
    for g in range(2):
        if g < len(grid):
            dd = grid[g]
            step = ext[dd] if ext[dd] else 1
            out += [math.log2(max(step * fu["strideA"][dd] * ELEM_BYTES[ta], 1)) / 40.0,
                    math.log2(max(step * fu["strideB"][dd] * ELEM_BYTES[tb], 1)) / 40.0]
        else:
            out += [0.0, 0.0]
    return kind + out


def candidate_features(p: Problem, tuning: dict, desc: dict, shape=None, groups=None) -> list[float]:
    head, mid, tail, nt, tile_bytes = shape or _shape_part(p, desc)
    t = desc.get("tile") or {}
    tv = tuning.get("tile_variant", 0)
    bl = tuning.get("blocks", 0)
    # the staged kernel's schedule: ring depth and CTAs per SM (the knobs, else the planner's),
    # and the bytes of tiles the whole GPU keeps in motion with them
    S = tuning.get("stages", 0) or t.get("stages", 3) or 3
    c = tuning.get("ctas_per_sm", 0) or t.get("ctas_per_sm", 0) or 4
    c = min(c, 4)
    ctas = bl if bl else c * 148
    W = ctas * (S - 1) * tile_bytes
    f = head + [1.0 if tv == 0 else 0.0, 1.0 if tv == 2 else 0.0, 1.0 if tv == 1 else 0.0,
                1.0 if bl == 0 else 0.0, bl / 444.0, S / 6.0, c / 4.0, math.log2(max(W, 1)) / 30.0] + mid
    waves = nt / ctas
    f += [math.log2(max(waves, 1e-3)) / 10.0, waves - math.floor(waves)] + tail
    # how the staged kernel moves the tiles: claimed in order or round robin; A runs shifted; bulk copies
    f += [1.0 if staged_claims(p, tuning, desc) else 0.0, float(t.get("shifted_runs", 0)), float(t.get("bulk", 0))]
    f += _raster_jumps(p, tuning, desc, groups)
    return f


def corpus_features(meta: dict) -> tuple[np.ndarray, np.ndarray]:
    """Recomputes the feature rows of a stored corpus from its cases and candidate tunings (shape-only
    planning on the host), so feature changes need no new measurements. Returns (X, case index)."""
    rows, case = [], []
    for c, tunings in zip(meta["cases"], meta["tunings"]):
        p = Problem(c["perm"], c["size"], c["dtype"], c.get("alpha", 1.0), c.get("beta", 0.0))
        descs = plan_shapes(p.perm, p.size, p.dtype, p.beta_nonzero, p.lda, p.ldb, tunings)
        X = features(p, list(zip(tunings, descs)))
        rows.append(X)
        case += [int(c["index"])] * len(X)
    return np.concatenate(rows).astype(np.float32), np.asarray(case, np.int32)


def features(p: Problem, cands) -> np.ndarray:
    """Feature matrix for [(tuning, plan json)] candidates of one problem."""
    if not cands:
        return np.zeros((0, 0), np.float32)
    pf = problem_features(p, cands[0][1])
    shapes = {}
    rows = []
    groups = None
    if any(tu.get("raster") for tu, _ in cands):
        from .autotune import fused_groups
        groups = fused_groups(p)[2]
    for tu, d in cands:
        sh = shapes.get(id(d))
        if sh is None:
            sh = shapes[id(d)] = _shape_part(p, d)
        rows.append(pf + candidate_features(p, tu, d, sh, groups))
    return np.asarray(rows, dtype=np.float32)


# ------------------------------------------------------------------------------------------------
def _lib():
    lib = _native.lib()
    if not hasattr(lib, "_mlp_bound"):
        P = ctypes.c_void_p
        I = ctypes.c_int
        F = ctypes.c_float
        lib.ttcb_mlp_gemm.argtypes = [I, I, I, I, I, P, I, P, I, P, I, P, I, P]
        lib.ttcb_mlp_relu_grad.argtypes = [P, P, P, I, P]
        lib.ttcb_mlp_colsum.argtypes = [P, I, I, P, P]
        lib.ttcb_mlp_mse.argtypes = [P, P, I, P, P, P]
        lib.ttcb_mlp_adam.argtypes = [P, P, P, P, I, F, F, F, F, I, P]
        lib.ttcb_mlp_adam_l2.argtypes = [P, P, P, P, I, F, F, F, F, F, I, P]
        for n in ("ttcb_mlp_gemm", "ttcb_mlp_relu_grad", "ttcb_mlp_colsum", "ttcb_mlp_mse", "ttcb_mlp_adam",
                  "ttcb_mlp_adam_l2"):
            getattr(lib, n).restype = ctypes.c_int
        lib._mlp_bound = True
    return lib


def _s():
    import torch
    return torch.cuda.current_stream().cuda_stream


def gemm(A, B, transA=False, transB=False, bias=None, relu=False, out=None):
    """op(A) @ op(B) (+bias) (relu) with the library's kernel; torch tensors hold the memory."""
    import torch
    M = A.shape[1] if transA else A.shape[0]
    K = A.shape[0] if transA else A.shape[1]
    N = B.shape[0] if transB else B.shape[1]
    C = out if out is not None else torch.empty((M, N), dtype=torch.float32, device=A.device)
    _native.check(_lib().ttcb_mlp_gemm(int(transA), int(transB), M, N, K, A.data_ptr(), A.shape[1], B.data_ptr(),
                                       B.shape[1], C.data_ptr(), N, bias.data_ptr() if bias is not None else None,
                                       int(relu), _s()))
    return C


class MLP:
    """Three dense layers (nin -> h -> h -> 1), ReLU between them, fp32 on the GPU."""

    def __init__(self, nin: int, hidden: int = 128, seed: int = 0):
        import torch
        g = np.random.default_rng(seed)

        def init(i, o):
            return torch.from_numpy((g.standard_normal((i, o)) * math.sqrt(2.0 / i)).astype(np.float32)).cuda()

        self.nin, self.hidden = nin, hidden
        self.params = [init(nin, hidden), torch.zeros(hidden, device="cuda"),
                       init(hidden, hidden), torch.zeros(hidden, device="cuda"),
                       init(hidden, 1) * 0.1, torch.zeros(1, device="cuda")]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.t = 0
        self.mu = np.zeros(nin, np.float32)
        self.sd = np.ones(nin, np.float32)
        self.ymu, self.ysd = 0.0, 1.0
        self.rmse = 1.0
        # further ensemble members (same shape and normalisation); predictions average over all
        self.extra = []

    def forward(self, X):
        W1, b1, W2, b2, W3, b3 = self.params
        H1 = gemm(X, W1, bias=b1, relu=True)
        H2 = gemm(H1, W2, bias=b2, relu=True)
        out = gemm(H2, W3, bias=b3)
        return out, (X, H1, H2)

    def backward(self, dout, cache):
        import torch
        X, H1, H2 = cache
        W1, b1, W2, b2, W3, b3 = self.params
        lib, s = _lib(), _s()
        grads = [None] * 6
        grads[4] = gemm(H2, dout, transA=True)
        grads[5] = torch.empty(1, device="cuda")
        _native.check(lib.ttcb_mlp_colsum(dout.data_ptr(), dout.shape[0], 1, grads[5].data_ptr(), s))
        dH2 = gemm(dout, W3, transB=True)
        dZ2 = torch.empty_like(dH2)
        _native.check(lib.ttcb_mlp_relu_grad(H2.data_ptr(), dH2.data_ptr(), dZ2.data_ptr(), dH2.numel(), s))
        grads[2] = gemm(H1, dZ2, transA=True)
        grads[3] = torch.empty(self.hidden, device="cuda")
        _native.check(lib.ttcb_mlp_colsum(dZ2.data_ptr(), dZ2.shape[0], dZ2.shape[1], grads[3].data_ptr(), s))
        dH1 = gemm(dZ2, W2, transB=True)
        dZ1 = torch.empty_like(dH1)
        _native.check(lib.ttcb_mlp_relu_grad(H1.data_ptr(), dH1.data_ptr(), dZ1.data_ptr(), dH1.numel(), s))
        grads[0] = gemm(X, dZ1, transA=True)
        grads[1] = torch.empty(self.hidden, device="cuda")
        _native.check(lib.ttcb_mlp_colsum(dZ1.data_ptr(), dZ1.shape[0], dZ1.shape[1], grads[1].data_ptr(), s))
        return grads

    def loss_grad(self, out, y):
        import torch
        d = torch.empty_like(out)
        loss = torch.zeros(1, device="cuda")
        _native.check(_lib().ttcb_mlp_mse(out.data_ptr(), y.data_ptr(), out.numel(), d.data_ptr(), loss.data_ptr(),
                                          _s()))
        return loss, d

    def step(self, grads, lr=1e-3, weight_decay=0.0):
        self.t += 1
        lib, s = _lib(), _s()
        for p, g, m, v in zip(self.params, grads, self.m, self.v):
            _native.check(lib.ttcb_mlp_adam_l2(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p.numel(),
                                               lr, 0.9, 0.999, 1e-8, weight_decay, self.t, s))

    # -- normalisation and I/O ------------------------------------------------------------------
    def _norm(self, X: np.ndarray):
        import torch
        return torch.from_numpy(((X - self.mu) / self.sd).astype(np.float32)).cuda()

    def predict(self, X: np.ndarray) -> np.ndarray:
        """Predicted log(GB/s) for each row of X (the mean over the ensemble's members)."""
        Xn = self._norm(X)
        out, _ = self.forward(Xn)
        acc = out.reshape(-1).clone()
        own = self.params
        for params in self.extra:
            self.params = params
            try:
                o, _ = self.forward(Xn)
            finally:
                self.params = own
            acc += o.reshape(-1)
        acc /= 1 + len(self.extra)
        return acc.cpu().numpy() * self.ysd + self.ymu

    def save(self, path: Path, extra: Optional[dict] = None):
        path.parent.mkdir(parents=True, exist_ok=True)
        arrays = {f"p{i}": p.cpu().numpy() for i, p in enumerate(self.params)}
        for k, params in enumerate(self.extra, start=1):
            arrays.update({f"m{k}_p{i}": p.cpu().numpy() for i, p in enumerate(params)})
        meta = {"version": VERSION, "nin": self.nin, "hidden": self.hidden, "ymu": self.ymu, "ysd": self.ysd,
                "rmse": self.rmse, "members": 1 + len(self.extra)}
        meta.update(extra or {})
        np.savez(path, mu=self.mu, sd=self.sd, meta=np.frombuffer(json.dumps(meta).encode(), np.uint8), **arrays)

    @classmethod
    def load(cls, path: Path) -> "MLP":
        import torch
        z = np.load(path)
        meta = json.loads(bytes(z["meta"]).decode())
        if meta.get("version") != VERSION:
            raise ValueError(f"cost model {path} has version {meta.get('version')}, expected {VERSION}")
        m = cls(meta["nin"], meta["hidden"])
        m.params = [torch.from_numpy(z[f"p{i}"]).cuda() for i in range(6)]
        m.extra = [[torch.from_numpy(z[f"m{k}_p{i}"]).cuda() for i in range(6)] for k in range(1, meta.get("members", 1))]
        m.mu, m.sd = z["mu"], z["sd"]
        m.ymu, m.ysd, m.rmse = meta["ymu"], meta["ysd"], meta["rmse"]
        m.meta = meta
        return m


def numpy_forward_backward(params, X, y):
    """CPU restatement (float64) of the same network's loss and gradients, for gradient checks."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(p, np.float64) for p in params]
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64).reshape(-1, 1)
    Z1 = X @ W1 + b1
    H1 = np.maximum(Z1, 0)
    Z2 = H1 @ W2 + b2
    H2 = np.maximum(Z2, 0)
    out = H2 @ W3 + b3
    n = out.size
    loss = float(np.mean((out - y) ** 2))
    d = 2 * (out - y) / n
    gW3 = H2.T @ d
    gb3 = d.sum(0)
    dH2 = d @ W3.T
    dZ2 = dH2 * (Z2 > 0)
    gW2 = H1.T @ dZ2
    gb2 = dZ2.sum(0)
    dH1 = dZ2 @ W2.T
    dZ1 = dH1 * (Z1 > 0)
    gW1 = X.T @ dZ1
    gb1 = dZ1.sum(0)
    return loss, [gW1, gb1, gW2, gb2, gW3, gb3]


def train(X: np.ndarray, y: np.ndarray, epochs: int = 60, lr: float = 2e-3, batch: int = 2048, seed: int = 0,
          val: float = 0.1, log=print, groups: Optional[np.ndarray] = None, members: int = 1,
          weight_decay: float = 0.0) -> MLP:
    """Fits log(GB/s) with the library's kernels. Holds out `val` of the rows for the RMSE (whole
    problems when `groups` gives each row's problem). With members > 1, trains that many networks
    from different initial weights on the same rows and returns them as one ensemble (predictions
    averaged). `weight_decay` is the L2 term of the Adam steps (on the normalised problem)."""
    import torch
    rng = np.random.default_rng(seed)
    val_groups = np.zeros(0, np.int64)
    if groups is not None:
        ug = rng.permutation(np.unique(groups))
        val_groups = ug[: int(len(ug) * val)]
        held = np.isin(groups, val_groups)
        vi, ti = np.nonzero(held)[0], rng.permutation(np.nonzero(~held)[0])
        nval = len(vi)
    else:
        idx = rng.permutation(len(X))
        nval = int(len(X) * val)
        vi, ti = idx[:nval], idx[nval:]
    m = MLP(X.shape[1], 128, seed)
    m.val_groups = val_groups
    m.mu = X[ti].mean(0)
    m.sd = X[ti].std(0) + 1e-6
    m.ymu, m.ysd = float(y[ti].mean()), float(y[ti].std() + 1e-6)
    Xt = m._norm(X[ti])
    yt = torch.from_numpy(((y[ti] - m.ymu) / m.ysd).astype(np.float32)).cuda().reshape(-1, 1)

    def fit(net: MLP, order_rng) -> float:
        """Trains one member; keeps the weights of its epoch with the lowest held-out error."""
        best_vr, best_params = float("inf"), None
        vr = float("nan")
        for ep in range(epochs):
            order = torch.from_numpy(order_rng.permutation(len(ti))).cuda()
            tot = 0.0
            for b0 in range(0, len(ti), batch):
                sel = order[b0:b0 + batch]
                xb, yb = Xt[sel].contiguous(), yt[sel].contiguous()
                out, cache = net.forward(xb)
                loss, d = net.loss_grad(out, yb)
                grads = net.backward(d, cache)
                net.step(grads, lr * (0.5 ** (ep // 20)), weight_decay)
                tot += float(loss.item()) * len(sel)
            if nval:
                vr = float(np.sqrt(np.mean((net.predict(X[vi]) - y[vi]) ** 2)))
                if vr < best_vr:
                    best_vr, best_params = vr, [q.clone() for q in net.params]
            if log and (ep % 10 == 0 or ep == epochs - 1):
                log(f"epoch {ep}: train mse {tot / len(ti):.4f} (normalised), val rmse {vr:.4f} log(GB/s)")
        if nval:
            net.params = best_params
        return best_vr

    fit(m, rng)
    for k in range(1, members):
        net = MLP(X.shape[1], 128, seed + k)
        net.mu, net.sd, net.ymu, net.ysd = m.mu, m.sd, m.ymu, m.ysd
        if log:
            log(f"member {k}")
        fit(net, np.random.default_rng(seed + 1000 * k))
        m.extra.append(net.params)
    if nval:
        m.rmse = float(np.sqrt(np.mean((m.predict(X[vi]) - y[vi]) ** 2)))
    return m


# ------------------------------------------------------------------------------------------------
def default_index(tunings: list) -> int:
    """Position of the planner's default schedule (the empty tuning) among candidate tunings."""
    for i, tu in enumerate(tunings):
        if not tu:
            return i
    return -1


def confidence_of(pred: np.ndarray, rmse: float) -> float:
    """1 - exp(-gap / rmse): gap = predicted log-GB/s margin of the best over the second-best."""
    if len(pred) < 2:
        return 1.0
    top = np.sort(pred)[::-1]
    return float(1.0 - math.exp(-(top[0] - top[1]) / max(rmse, 1e-6)))


_loaded = {}


def load_default(path: Optional[Path] = None) -> MLP:
    path = Path(path or DEFAULT_MODEL)
    if str(path) not in _loaded:
        _loaded[str(path)] = MLP.load(path)
    return _loaded[str(path)]


# The selection policy. The planner's default is within a few percent of the exhaustive search's
# winner for most problems, so the network's choice is only taken on a predicted gain over the
# default: at least POLICY["hi"] (log GB/s), its top-1 untimed; between POLICY["lo"] and
# POLICY["hi"], its top POLICY["k"] candidates and the default are timed and the fastest kept; below
# POLICY["lo"] the default stays. On the 500 held-out problems' stored timings, timing the top 1, 2
# or 3 with the default kept 0.952, 0.964 and 0.971 of the best measured GB/s (the default alone
# 0.925). `train` fits the thresholds on its held-out problems and stores them with the model.
DEFAULT_POLICY = {"lo": 0.02, "hi": 0.3, "k": 2}  # a trained model stores its own (lo, hi, k)


def policy_of(model) -> dict:
    return dict(DEFAULT_POLICY, **(getattr(model, "meta", {}) or {}).get("policy", {}))


def decide(pred: np.ndarray, default: int, policy: dict) -> tuple[list, bool]:
    """(candidate indices to use, timed?) for one problem's predictions under the policy: one index
    when the choice is made without timing, the network's top k and the default when they are to be
    timed."""
    top = int(np.argmax(pred))
    if default < 0:
        return [top], False
    if top == default:
        return [default], False
    gain = float(pred[top] - pred[default])
    if gain >= policy["hi"]:
        return [top], False
    if gain >= policy["lo"]:
        k = max(int(policy.get("k", 1)), 1)
        picks = [int(i) for i in np.argsort(-pred) if int(i) != default][:k]
        return picks + [default], True
    return [default], False


def select(p: Problem, max_impl: int = 64, confidence: Optional[float] = None, verify: bool = True,
           model: Optional[MLP] = None, measure_choice: bool = True) -> dict:
    """Picks a schedule with the model under its policy (see DEFAULT_POLICY); `confidence=0.0` takes
    the network's top-1 untimed whatever it predicts. Returns the measured results of the timed
    candidates (or of the choice, with measure_choice)."""
    model = model or load_default()
    t0 = time.perf_counter()
    cands = candidate_tunings(p, max_impl, with_desc=True)
    X = features(p, cands)
    pred = model.predict(X)
    order = np.argsort(-pred)
    conf = confidence_of(pred, model.rmse)
    d = default_index([c[0] for c in cands])
    if confidence == 0.0:
        picks, timed = [int(order[0])], False
    else:
        picks, timed = decide(pred, d, policy_of(model))
    chosen = [cands[i][0] for i in picks]
    t_model = time.perf_counter() - t0
    results = measure(p, chosen, reps=3, verify=verify) if (measure_choice or timed) else []
    return {"results": results, "confidence": conf, "fallback": timed, "pred": pred, "order": order,
            "picks": picks, "candidates": cands, "seconds_model": t_model, "seconds": time.perf_counter() - t0}


def fresh_head_to_head(cases: list[dict], model: Optional[MLP] = None, max_impl: int = 64, reps: int = 5) -> dict:
    """The selector against the method without it, on fresh timings: per problem, every candidate
    is timed (the exhaustive search, TTC's method), then the search's winner, the network's top-1,
    the selector's choice (under the model's policy: the default, the top-1, or the fastest of its top
    k and the default, timed) and the planner default are re-timed alternately, so the winner loses the bias of being the
    maximum of noisy timings. Returns the mean shares of the winner's GB/s and the tuning times."""
    from .autotune import search
    model = model or load_default()
    rows = []
    if cases:
        # first use of the model, the kernels and the timing buffers, outside the timed comparison
        c = cases[0]
        p = Problem(c["perm"], c["size"], c["dtype"], c.get("alpha", 1.0), c.get("beta", 0.0))
        search(p, max_impl=2, reps=1, verify=False)
        select(p, max_impl=max_impl, model=model, verify=False, measure_choice=True)
    for c in cases:
        p = Problem(c["perm"], c["size"], c["dtype"], c.get("alpha", 1.0), c.get("beta", 0.0))
        sr = search(p, max_impl=max_impl, reps=3, verify=False)
        top = select(p, max_impl=max_impl, confidence=0.0, model=model, verify=False, measure_choice=False)
        sel = select(p, max_impl=max_impl, model=model, verify=False, measure_choice=False)
        top1 = top["candidates"][int(top["order"][0])][0]
        chosen = (min(sel["results"], key=lambda r: r.time_ms).tuning if sel["results"]
                  else sel["candidates"][sel["picks"][0]][0])
        picks = [sr["best"].tuning, top1, chosen, {}]
        bench = Bench(p, seed=1)
        best_ms = [float("inf")] * len(picks)
        for rnd in range(2):
            order = list(range(len(picks))) if rnd == 0 else list(reversed(range(len(picks))))
            for i, r in zip(order, measure(p, [picks[i] for i in order], reps=reps, verify=False, bench=bench)):
                best_ms[i] = min(best_ms[i], r.time_ms)
        del bench
        rows.append({"search_s": sr["seconds"], "top1_s": top["seconds"], "sel_s": sel["seconds"],
                     "top1": best_ms[0] / best_ms[1], "sel": best_ms[0] / best_ms[2], "dflt": best_ms[0] / best_ms[3],
                     "fallback": bool(sel["fallback"])})
    m = lambda k: float(np.mean([r[k] for r in rows]))
    return {"problems": len(rows), "search_candidates": max_impl,
            "top1_over_search": round(m("top1"), 4), "selector_over_search": round(m("sel"), 4),
            "default_over_search": round(m("dflt"), 4),
            "selector_within_5pct": round(float(np.mean([r["sel"] >= 0.95 for r in rows])), 4),
            "top1_within_5pct": round(float(np.mean([r["top1"] >= 0.95 for r in rows])), 4),
            "fallbacks": int(sum(r["fallback"] for r in rows)),
            "search_seconds_mean": round(m("search_s"), 3), "selector_seconds_mean": round(m("sel_s"), 4),
            "top1_seconds_mean": round(m("top1_s"), 4),
            "tuning_time_ratio_selector": round(m("search_s") / max(m("sel_s"), 1e-9), 1),
            "tuning_time_ratio_top1": round(m("search_s") / max(m("top1_s"), 1e-9), 1),
            "timing": f"fresh: winner, top-1, selector choice and default re-timed alternately, best of 2x{reps} launches"}


# seeds of the training problems and of the held-out problems (ttc_b200.workloads.learning_cases)
TRAIN_SEED = 11
HELDOUT_SEED = 12345


def choose_tuning(p: Problem, model: Optional[MLP] = None) -> Optional[dict]:
    """The learned selector's schedule for one problem, as the benchmark uses it: under the model's
    policy, the planner default, the network's top-1, or the fastest of its top k and the default
    (timed on the GPU with the problem's own inputs). None means the planner default."""
    sel = select(p, verify=False, measure_choice=False, model=model)
    if sel["results"]:
        tu = min(sel["results"], key=lambda r: r.time_ms).tuning
    else:
        tu = sel["candidates"][sel["picks"][0]][0]
    return tu or None


# ------------------------------------------------------------------------------------------------
def collect(cases: list[dict], out: Path, max_impl: int = 64, reps: int = 3, log=print,
            deadline: Optional[float] = None) -> bool:
    """Exhaustive measured search over each case's candidates; stores features, log(GB/s), the
    search wall time, resumable per case (rows of finished cases are kept). Stops early, keeping
    what it has, once time.time() passes `deadline`; returns True when every case is done."""
    import torch
    done = {}
    if out.exists():
        z = np.load(out, allow_pickle=False)
        done = {"X": list(z["X"]), "y": list(z["y"]), "case": list(z["case"]), "cand": list(z["cand"]),
                "search_s": list(z["search_s"]), "meta": json.loads(bytes(z["meta"]).decode())}
    else:
        done = {"X": [], "y": [], "case": [], "cand": [], "search_s": [], "meta": {"cases": [], "tunings": []}}
    finished = {int(c) for c in done["case"]}
    t_last = time.time()
    for k, c in enumerate(cases):
        if k in finished:
            continue
        if deadline is not None and time.time() > deadline:
            _save_corpus(out, done)
            return False
        p = Problem(c["perm"], c["size"], c["dtype"], c.get("alpha", 1.0), c.get("beta", 0.0))
        t0 = time.perf_counter()
        cands = candidate_tunings(p, max_impl, with_desc=True)
        res = measure(p, [tu for tu, _ in cands], reps=reps, verify=True, seed=k)
        secs = time.perf_counter() - t0
        if not all(r.ok for r in res):
            raise RuntimeError(f"schedules disagree on case {k}: {c}")
        X = features(p, cands)
        for j, r in enumerate(res):
            done["X"].append(X[j])
            done["y"].append(math.log(max(r.gbs, 1e-3)))
            done["case"].append(k)
            done["cand"].append(j)
        done["search_s"].append(secs)
        done["meta"]["cases"].append(dict(c, index=k))
        done["meta"]["tunings"].append([tu for tu, _ in cands])
        torch.cuda.empty_cache()
        if time.time() - t_last > 60 or k == len(cases) - 1:
            _save_corpus(out, done)
            t_last = time.time()
            if log:
                log(f"collected {k + 1}/{len(cases)} cases, {len(done['y'])} rows")
    _save_corpus(out, done)
    return True


def _save_corpus(out: Path, d: dict):
    out.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out, X=np.asarray(d["X"], np.float32), y=np.asarray(d["y"], np.float32),
             case=np.asarray(d["case"], np.int32), cand=np.asarray(d["cand"], np.int32),
             search_s=np.asarray(d["search_s"], np.float64),
             meta=np.frombuffer(json.dumps(d["meta"]).encode(), np.uint8))


def stored_selection(pred: np.ndarray, y: np.ndarray, case: np.ndarray, meta: dict, policy: dict) -> dict:
    """Selection quality on stored exhaustive measurements: per problem, the GB/s of the model's
    top-1, of the policy's choice (when it times the top-1 and the default, the faster by the stored
    timings) and of the planner's default schedule, each over the best measured GB/s."""
    index_of = {int(c["index"]): i for i, c in enumerate(meta["cases"])}
    top1, gated, dflt, fb = [], [], [], []
    for k in np.unique(case):
        rows = np.nonzero(case == k)[0]
        tunings = meta["tunings"][index_of[int(k)]]
        best = y[rows].max()
        top1.append(np.exp(y[rows[int(np.argmax(pred[rows]))]] - best))
        d = tunings.index({}) if {} in tunings else 0
        picks, timed = decide(pred[rows], d, policy)
        fb.append(timed)
        gated.append(np.exp(y[rows[picks]].max() - best))
        dflt.append(np.exp(y[rows[d]] - best))
    top1, gated, dflt = map(np.asarray, (top1, gated, dflt))
    return {"cases": int(len(top1)), "top1_over_best": float(top1.mean()),
            "top1_within_5pct": float(np.mean(top1 >= 0.95)), "gated_over_best": float(gated.mean()),
            "gated_within_5pct": float(np.mean(gated >= 0.95)), "timed_fraction": float(np.mean(fb)),
            "default_over_best": float(dflt.mean()), "default_within_5pct": float(np.mean(dflt >= 0.95)),
            "gain_over_default": float(np.mean(gated / dflt))}


def fit_policy(pred: np.ndarray, y: np.ndarray, case: np.ndarray, meta: dict, timing_cost: float = 0.005) -> dict:
    """The policy (thresholds and candidates timed) that keeps the largest share of the best GB/s on
    these problems, less `timing_cost` per candidate timed per problem (the policy's tuning time)."""
    best, best_score = dict(DEFAULT_POLICY), -1e9
    for k in (1, 2, 3):
        for lo in (0.0, 0.01, 0.02, 0.05, 0.1, 0.2, float("inf")):
            for hi in (0.05, 0.1, 0.2, 0.3, 0.5, 1.0, float("inf")):
                if hi < lo:
                    continue
                pol = {"lo": lo, "hi": hi, "k": k}
                r = stored_selection(pred, y, case, meta, pol)
                score = r["gated_over_best"] - timing_cost * (k + 1) * r["timed_fraction"]
                if score > best_score + 1e-9:
                    best, best_score = pol, score
    return best


def evaluate(model: MLP, corpus: Path, log=print, time_cases: int = 100, fresh_cases: int = 40) -> dict:
    """Held-out evaluation.

    1. Stored measurements (every held-out problem): the model's top-1, the policy's choice and the
       planner default, each over the best GB/s of the exhaustive search, and the same for a grid of
       policy thresholds.
    2. Fresh head to head (first `fresh_cases` problems, fresh_head_to_head): the search is run
       again and its winner, the top-1, the policy's choice and the default re-timed alternately.
    3. Tuning time (first `time_cases` problems): the exhaustive search's recorded wall time
       against the model's (candidate planning, features, GPU inference, and the two timings when
       the policy times)."""
    z = np.load(corpus)
    y, case = z["y"], z["case"]
    meta = json.loads(bytes(z["meta"]).decode())
    X, _ = corpus_features(meta)
    pred = model.predict(X)
    pol = policy_of(model)
    res = {"policy": pol, "stored": stored_selection(pred, y, case, meta, pol),
           "stored_curve": [dict(lo=lo, hi=hi, **{k: v for k, v in stored_selection(
               pred, y, case, meta, {"lo": lo, "hi": hi}).items() if k in ("gated_over_best", "timed_fraction")})
                            for lo in (0.0, 0.02, 0.05, 0.1) for hi in (0.1, 0.3, 1.0)]}
    cases = meta["cases"]
    search_s = z["search_s"]
    if fresh_cases:
        res["fresh"] = fresh_head_to_head(cases[:fresh_cases], model)

    # tuning time
    t_top1, t_gated, t_search, fbs = [], [], [], 0
    for i, c in enumerate(cases[:time_cases]):
        p = Problem(c["perm"], c["size"], c["dtype"], c.get("alpha", 1.0), c.get("beta", 0.0))
        r = select(p, confidence=0.0, model=model, verify=False, measure_choice=False)
        t_top1.append(r["seconds"])
        r = select(p, model=model, verify=False, measure_choice=False)
        t_gated.append(r["seconds"])
        fbs += int(r["fallback"])
        t_search.append(search_s[i])
    res["time"] = {"cases": len(t_search), "search_seconds_mean": float(np.mean(t_search)),
                   "model_top1_seconds_mean": float(np.mean(t_top1)),
                   "model_policy_seconds_mean": float(np.mean(t_gated)),
                   "top1_speedup": float(np.mean(t_search) / max(np.mean(t_top1), 1e-9)),
                   "policy_speedup": float(np.mean(t_search) / max(np.mean(t_gated), 1e-9)),
                   "policy_timed": fbs}
    res["rmse"] = model.rmse
    if log:
        log(json.dumps(res, indent=1))
    return res


def main(argv=None):
    import ttc_b200.workloads as wl
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["collect", "train", "evaluate"])
    ap.add_argument("--train-cases", type=int, default=2000)
    ap.add_argument("--test-cases", type=int, default=500)
    ap.add_argument("--corpus", default=str(Path(__file__).resolve().parent / "data" / "cost_corpus"),
                    help="corpus path prefix (<prefix>_train.npz, <prefix>_test.npz)")
    ap.add_argument("--model", default=str(DEFAULT_MODEL))
    ap.add_argument("--max-impl", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--members", type=int, default=1, help="train: networks in the ensemble")
    ap.add_argument("--weight-decay", type=float, default=0.0,
                    help="train: L2 weight decay of the Adam steps. 1e-3 lowered the held-out RMSE (0.274 to "
                         "0.238 log GB/s) but not the fresh selection: its untimed top-1 kept less of the "
                         "search winner's GB/s, so the shipped model is trained without it")
    ap.add_argument("--out-json", default=None)
    ap.add_argument("--max-seconds", type=float, default=None, help="collect: stop (resumably) after this long")
    a = ap.parse_args(argv)
    train_path = Path(a.corpus + "_train.npz")
    test_path = Path(a.corpus + "_test.npz")
    if a.cmd == "collect":
        deadline = time.time() + a.max_seconds if a.max_seconds else None
        if collect(wl.learning_cases(TRAIN_SEED, a.train_cases), train_path, a.max_impl, deadline=deadline):
            collect(wl.learning_cases(HELDOUT_SEED, a.test_cases), test_path, a.max_impl, deadline=deadline)
    elif a.cmd == "train":
        z = np.load(train_path)
        X, case = corpus_features(json.loads(bytes(z["meta"]).decode()))
        meta = json.loads(bytes(z["meta"]).decode())
        m = train(X, z["y"], epochs=a.epochs, groups=case, members=a.members, weight_decay=a.weight_decay)
        # the policy thresholds, fitted on the training run's held-out problems
        held = np.isin(case, m.val_groups)
        policy = fit_policy(m.predict(X[held]), z["y"][held], case[held], meta) if held.any() else DEFAULT_POLICY
        digest = hashlib.sha256(z["X"].tobytes()[:1 << 20]).hexdigest()[:16]
        m.save(Path(a.model), {"trained_rows": int(len(z["y"])), "corpus_digest": digest, "policy": policy,
                               "members": a.members, "weight_decay": a.weight_decay, "epochs": a.epochs})
        print(f"saved {a.model} (val rmse {m.rmse:.4f}, policy {policy})")
    else:
        m = MLP.load(Path(a.model))
        res = evaluate(m, test_path)
        if a.out_json:
            Path(a.out_json).write_text(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
