"""Seeded synthetic workloads (shapes, permutations, scalars) for the
benchmarks and the full-size tests.  No data: callers fill tensors.

* plain_single()  f32 {256,256,256}, perm {2,1,0}, alpha 2.3, beta 4.2
* sweep_cases()   48 cases over ranks 2-6 in f32/f64, random non-identity
                  perms, extents log-uniform in [4, 4096] rescaled so each
                  tensor holds ~200 MB (extents may exceed 4096 after the
                  rescale: a rank-2 f32 tensor of 200 MB needs ~7071 per dim)
* hard_cases()    c64/c128 rank 6, stride-1 extents 2-16, ~256 MB per tensor
* batch_cases()   4096 mixed transposes, 4 KB - 16 MB each (~6 GB in total)
* contraction_cases()  tensor contractions for the transpose-GEMM-transpose
                  path: 1-3 M, N and K labels, 0-1 batch labels, random label
                  orders in every tensor, GEMM extents m, n ~ 1-4 K, k ~ 0.5-2 K
"""
from __future__ import annotations

import math
from typing import Dict, List

import numpy as np

ELEM = {"f32": 4, "f64": 8, "c64": 8, "c128": 16}


def _perm(rng, rank, non_identity=True) -> List[int]:
    while True:
        p = [int(x) for x in rng.permutation(rank)]
        if not non_identity or p != list(range(rank)):
            return p


def _rescale(ext: List[float], target: float, lo: int = 1) -> List[int]:
    rank = len(ext)
    prod = float(np.prod(ext))
    s = (target / prod) ** (1.0 / rank)
    out = [max(lo, int(round(e * s))) for e in ext]
    # correct the largest dim so the element count lands near the target
    cur = float(np.prod(out))
    j = int(np.argmax(out))
    out[j] = max(lo, int(round(out[j] * target / cur)))
    return out


def plain_single() -> Dict:
    return {"dtype": "f32", "in_size": [256, 256, 256], "perm": [2, 1, 0],
            "alpha": 2.3, "beta": 4.2, "seed": 0}


def sweep_cases(seed: int = 2024, tensor_bytes: float = 200e6) -> List[Dict]:
    rng = np.random.default_rng(seed)
    counts = {2: 10, 3: 10, 4: 10, 5: 9, 6: 9}
    cases = []
    i = 0
    for rank, cnt in counts.items():
        for _ in range(cnt):
            dtype = "f32" if i % 2 == 0 else "f64"
            ext = list(np.exp(rng.uniform(math.log(4), math.log(4096), rank)))
            size = _rescale(ext, tensor_bytes / ELEM[dtype], lo=4)
            cases.append({"dtype": dtype, "in_size": size, "perm": _perm(rng, rank)})
            i += 1
    return cases


def hard_cases() -> List[Dict]:
    out = []
    for dtype, size in (("c64", [8, 64, 4, 64, 16, 16]), ("c128", [8, 64, 4, 64, 16, 8])):
        for perm in ([5, 2, 0, 4, 1, 3], [0, 3, 2, 1, 4, 5]):
            out.append({"dtype": dtype, "in_size": list(size), "perm": list(perm),
                        "alpha": complex(1.5, -0.5), "beta": complex(0.25, 1.0)})
    return out


def batch_cases(count: int = 4096, seed: int = 7, lo_bytes: float = 4096,
                hi_bytes: float = 16 * 2 ** 20) -> List[Dict]:
    rng = np.random.default_rng(seed)
    names = ["f32", "f64", "c64", "c128"]
    cases = []
    for _ in range(count):
        dtype = names[int(rng.integers(0, 4))]
        rank = int(rng.integers(2, 7))
        nbytes = math.exp(rng.uniform(math.log(lo_bytes), math.log(hi_bytes)))
        target = max(1.0, nbytes / ELEM[dtype])
        ext = list(np.exp(rng.uniform(0, math.log(64), rank)))
        size = _rescale(ext, target, lo=1)
        perm = _perm(rng, rank, non_identity=True)
        if rng.random() < 0.5:
            alpha, beta = 1.0, 0.0
        elif dtype in ("c64", "c128"):
            alpha = complex(rng.uniform(-2, 2), rng.uniform(-2, 2))
            beta = complex(rng.uniform(-2, 2), rng.uniform(-2, 2))
        else:
            alpha, beta = float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2))
        cases.append({"dtype": dtype, "in_size": size, "perm": perm,
                      "alpha": alpha, "beta": beta})
    return cases


def _split(rng, total: float, parts: int) -> List[int]:
    """Extents of `parts` labels whose product is about `total`."""
    if parts == 0:
        return []
    w = rng.uniform(0.5, 1.5, parts)
    ext = [max(2, int(round(total ** (x / w.sum())))) for x in w]
    return ext


def contraction_cases(count: int = 8, seed: int = 11) -> List[Dict]:
    """Seeded synthetic contractions C[lc] = alpha * A[la] B[lb] + beta * C:
    f32 and f64 (one c64 and one c128), label orders drawn at random, so most
    operands need a transpose before the GEMM and most outputs one after."""
    rng = np.random.default_rng(seed)
    names = ["f32", "f64", "f32", "f64", "f32", "f64", "c64", "c128"]
    letters = "abcdefghijklmnop"
    cases = []
    for i in range(count):
        dtype = names[i % len(names)]
        cplx = dtype in ("c64", "c128")
        nm, nn, nk = (int(rng.integers(1, 4)) for _ in range(3))
        nb = int(rng.integers(0, 2))
        lab = iter(letters)
        M = [next(lab) for _ in range(nm)]
        N = [next(lab) for _ in range(nn)]
        K = [next(lab) for _ in range(nk)]
        Bt = [next(lab) for _ in range(nb)]
        scale = 0.5 if cplx else 1.0
        m = math.exp(rng.uniform(math.log(1024), math.log(4096))) * scale
        n = math.exp(rng.uniform(math.log(1024), math.log(4096))) * scale
        k = math.exp(rng.uniform(math.log(512), math.log(2048))) * scale
        bsz = 4 if nb else 1
        ext = dict(zip(M, _split(rng, m / bsz ** 0.5, nm)))
        ext.update(zip(N, _split(rng, n / bsz ** 0.5, nn)))
        ext.update(zip(K, _split(rng, k, nk)))
        ext.update(zip(Bt, [bsz] * nb))
        la = [str(x) for x in rng.permutation(M + K + Bt)]
        lb = [str(x) for x in rng.permutation(K + N + Bt)]
        lc = [str(x) for x in rng.permutation(M + N + Bt)]
        alpha, beta = (1.0, 0.0) if i % 2 == 0 else (0.5, -1.5)
        cases.append({"dtype": dtype, "labels_a": la, "labels_b": lb, "labels_c": lc,
                      "size_a": [ext[x] for x in la], "size_b": [ext[x] for x in lb],
                      "size_c": [ext[x] for x in lc], "alpha": alpha, "beta": beta})
    return cases


def algorithmic_bytes(case: Dict, beta=None) -> int:
    """2*N*sizeof(T), plus N*sizeof(T) when B is read (|beta| >= 1e-16)."""
    n = int(np.prod(case["in_size"]))
    b = case.get("beta", 0.0) if beta is None else beta
    reads_b = abs(complex(b).real) >= 1e-16 or abs(complex(b).imag) >= 1e-16
    return n * ELEM[case["dtype"]] * (3 if reads_b else 2)
