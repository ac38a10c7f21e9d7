"""TTC's argument object and helpers, with the same names and meaning (ttc_util.py in the TTC project).

`TTCargs` carries the same fields as TTC's (ttc_util.py:46-115) plus `model`, `confidence` and
`batched` for the learned selector and batched mode. Type names follow TTC: "float", "double",
"float complex", "double complex".
"""
from __future__ import annotations

import copy
import math
from typing import List

OKGREEN = "\033[92m"
FAIL = "\033[91m"
WARNING = "\033[93m"
ENDC = "\033[0m"

FLOAT_TYPE_SIZE = {"float": 4, "double": 8, "float complex": 8, "double complex": 16}
PREFIX = {("float", "float"): "s", ("double", "double"): "d", ("double", "float"): "ds", ("float", "double"): "sd",
          ("float complex", "float complex"): "c", ("double complex", "double complex"): "z",
          ("double complex", "float complex"): "zc", ("float complex", "double complex"): "cz"}
TYPES_OF_PREFIX = {v: k for k, v in PREFIX.items()}


def getVersion():
    return [0, 1, 2]


def getFloatTypeSize(floatType: str) -> int:
    """Bytes of one element (ttc_util.py:23-34). Raises ValueError for an unknown type."""
    if floatType not in FLOAT_TYPE_SIZE:
        raise ValueError("[TTC] ERROR: unknown data type")
    return FLOAT_TYPE_SIZE[floatType]


def getFloatPrefix(floatTypeA: str, floatTypeB: str) -> str:
    """TTC's --dataType letters for a type pair (ttc_util.py:117-133)."""
    return PREFIX[(floatTypeA, floatTypeB)]


def listToString(l) -> str:
    return "(" + ",".join(str(x) for x in l) + ")" if len(l) else ""


class TTCargs:
    """Arguments of one transposition (ttc_util.py:46-115); same fields, same defaults."""

    def __init__(self, idxPerm, size):
        self.size = copy.deepcopy(list(size))
        self.idxPerm = copy.deepcopy(list(idxPerm))
        self.alpha = 1.
        self.keep = 0
        self.generateOnly = 0
        self.beta = 0.
        self.affinity = ""
        self.numThreads = 0
        self.floatTypeA = "float"
        self.floatTypeB = "float"
        self.streamingStores = 0
        self.maxNumImplementations = 200
        self.lda: List[int] = []
        self.ldb: List[int] = []
        self.debug = 0
        self.architecture = "avx"
        self.align = 1
        self.blockings = []
        self.loopPermutations = []
        self.prefetchDistances = []
        self.scalar = 0
        self.silent = 0
        self.ignoreDatabase = 0
        self.compiler = "icpc"
        self.hostName = ""
        self.vecLength = []
        self.hotA = 0
        self.hotB = 0
        self.updateDatabase = 1
        # additions of this implementation
        self.noTest = 0
        self.model = 0            # 1: rank candidates with the learned cost model
        self.confidence = 0.0     # measured-search fallback below this model confidence (0 = default)
        self.batched = 0

    def getSize(self):
        return copy.deepcopy(self.size)

    def getPerm(self):
        return copy.deepcopy(self.idxPerm)

    def dataType(self) -> str:
        return getFloatPrefix(self.floatTypeA, self.floatTypeB)

    def getCommandLineString(self) -> str:
        s = (f"ttc --beta={self.beta:f} --perm={','.join(map(str, self.idxPerm))} "
             f"--size={','.join(map(str, self.size))} --architecture={self.architecture} "
             f"--maxImplementations={self.maxNumImplementations}")
        if self.lda:
            s += f" --lda={','.join(map(str, self.lda))}"
        if self.ldb:
            s += f" --ldb={','.join(map(str, self.ldb))}"
        s += f" --compiler={self.compiler} --dataType={self.dataType()} --numThreads={self.numThreads}"
        if self.streamingStores:
            s += " --streamingStores"
        return s


def getCostLoop(loopPerm, perm, size) -> float:
    """TTC's loop-order cost (ttc_util.py:167-209): sum over loops of trip count times the squared
    jump distances in A and B when the loop advances. Lower is better."""
    n = len(size)
    lda = [1] * n
    ldb = [1] * n
    for i in range(1, n):
        lda[i] = lda[i - 1] * size[i - 1]
        ldb[i] = ldb[i - 1] * size[perm[i - 1]]
    pos_in_b = {p: j for j, p in enumerate(perm)}
    total, cost = 1, 0.0
    for i, d in enumerate(loopPerm):
        last_a = sum(lda[e] * (size[e] - 1) for e in loopPerm[i + 1:])
        last_b = sum(ldb[pos_in_b[e]] * (size[e] - 1) for e in loopPerm[i + 1:])
        cost += total * (size[d] - 1) * ((last_a - lda[d]) ** 2.0 + (last_b - ldb[pos_in_b[d]]) ** 2.0)
        total *= size[d]
    return cost


def fuseIndices(size, perm, loopPermutations, lda, ldb):
    """In-place index fusion with TTC's semantics (ttc_util.py:214-276): runs of A-dims that stay
    consecutive in B and are unpadded become one dimension; loop orders are renumbered. An empty
    lda (ldb) means dense: the fusion then works on a local dense copy and the caller's list stays
    empty, as in TTC, whose generators fill the dense defaults from the fused sizes
    (GPUtransposeGenerator.py:87-94)."""
    if len(lda) == 0:
        lda = list(size)
    if len(ldb) == 0:
        ldb = [size[p] for p in perm]
    idx = list(range(len(size)))
    i = 0
    while i < len(idx):
        for j in range(len(perm)):
            run, total = 0, 1
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
    order = sorted(range(len(perm)), key=lambda k: perm[k])
    newperm = [0] * len(perm)
    for r, k in enumerate(order):
        newperm[k] = r
    perm[:] = newperm
    for loopOrder in loopPermutations:
        diff = len(loopOrder) - len(perm)
        for k in range(len(loopOrder)):
            loopOrder[k] -= diff
        loopOrder[:] = [x for x in loopOrder if x >= 0]


def denseLeadingDims(size, perm, lda, ldb):
    """lda/ldb with TTC's dense defaults filled in (lda = size, ldb[j] = size[perm[j]]) where the
    caller left them empty (GPUtransposeGenerator.py:87-94)."""
    return (list(lda) if len(lda) else list(size)), (list(ldb) if len(ldb) else [size[p] for p in perm])


def streamingStoresApplicable(ldb, size, perm, beta, alignmentRequirementBytes, floatSizeBytes, useStreamingStores):
    """TTC's rule (ttc_util.py:301-314); on the GPU, streaming stores are used whenever beta == 0."""
    leading = ldb[0] if len(ldb) else size[perm[0]]
    if useStreamingStores == 1 and beta == 0:
        if perm[0] == 0:
            return 1
        return 1 if (leading * floatSizeBytes) % alignmentRequirementBytes == 0 else 0
    return 0


def getArchitecture(arch: str) -> str:
    """Name of the device the measurements belong to (ttc_util.py:145-165 reads `nvidia-smi -L`)."""
    if arch == "cuda":
        try:
            import torch
            if torch.cuda.is_available():
                return " " + torch.cuda.get_device_name(torch.cuda.current_device())
        except Exception:
            pass
        return " unknown CUDA device"
    return "host"


def elements(size) -> int:
    return math.prod(size) if len(size) else 0
