"""TEST INFRASTRUCTURE - Python restatements of TTC's planning helpers, used as checkers.

* ``fuse_indices``   - TTC's index fusion (ttc_util.py:214-276 in the TTC project): runs of
  A-dimensions that appear in the same consecutive order in B, and are unpadded (lda[k] == size[k],
  ldb[j] == size[k] for the inner dimension of a merged pair), become one dimension.
* ``cost_loop``      - TTC's loop-order cost (ttc_util.py:167-209): sum over loops of
  (trip count) * (squared jump distance in A + squared jump distance in B).
* ``strides``        - strides from the outer-size convention (CUDAtranspose.py:543-556).
"""
from __future__ import annotations


def strides(size, perm, lda=None, ldb=None):
    """Returns (strideA per A-dim, strideB per A-dim) in elements."""
    n = len(size)
    la = list(lda) if lda else list(size)
    lb = list(ldb) if ldb else [size[p] for p in perm]
    sA = [1] * n
    sBpos = [1] * n
    for i in range(1, n):
        sA[i] = sA[i - 1] * la[i - 1]
        sBpos[i] = sBpos[i - 1] * lb[i - 1]
    sB = [0] * n
    for j, p in enumerate(perm):
        sB[p] = sBpos[j]
    return sA, sB


def fuse_indices(size, perm, lda=None, ldb=None):
    """TTC's fusion. Returns (size, perm, lda, ldb) after fusion (new lists)."""
    size = list(size)
    perm = list(perm)
    lda = list(lda) if lda else list(size)
    ldb = list(ldb) if ldb else [size[p] for p in perm]
    idx = list(range(len(size)))
    i = 0
    while i < len(idx):
        for j in range(len(perm)):
            run = 0
            total = 1
            while (i + run < len(idx) and j + run < len(perm) and idx[i + run] == perm[j + run]
                   and (run == 0 or lda[i + run - 1] == size[i + run - 1])
                   and (run == 0 or ldb[j + run - 1] == size[i + run - 1])):
                total *= size[i + run]
                run += 1
            if run >= 1:
                size[i] = total
            while run > 1:
                idx.pop(i + 1)
                perm.pop(j + 1)
                size.pop(i + 1)
                lda[i] *= lda[i + 1]
                lda.pop(i + 1)
                ldb[j] *= ldb[j + 1]
                ldb.pop(j + 1)
                run -= 1
        i += 1
    # close the gaps in the numbering (e.g. [0,1,3] -> [0,1,2])
    order = sorted(range(len(perm)), key=lambda k: perm[k])
    newperm = [0] * len(perm)
    for rank_, k in enumerate(order):
        newperm[k] = rank_
    return size, newperm, lda, ldb


def cost_loop(loop_perm, perm, size):
    """TTC's loop-order cost: lower is better."""
    n = len(size)
    lda = [1] * n
    ldb = [1] * n
    for i in range(1, n):
        lda[i] = lda[i - 1] * size[i - 1]
        ldb[i] = ldb[i - 1] * size[perm[i - 1]]
    inv = {p: j for j, p in enumerate(perm)}
    total = 1
    cost = 0.0
    for i, d in enumerate(loop_perm):
        last_a = 0
        last_b = 0
        for d2 in loop_perm[i + 1:]:
            last_a += lda[d2] * (size[d2] - 1)
            last_b += ldb[inv[d2]] * (size[d2] - 1)
        cost += total * (size[d] - 1) * ((last_a - lda[d]) ** 2.0 + (last_b - ldb[inv[d]]) ** 2.0)
        total *= size[d]
    return cost
