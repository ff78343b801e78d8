"""Generate tests/golden/golden.npz from the reference's own CPU code.

Run here (where the reference sources exist and oracle/_ref is built):

    make -C oracle ref && python tests/golden/make_golden.py

Each case holds A, B before, B after, and the call's arguments.  Cases on
which the reference plan is correct (see oracle.ref_plan_is_safe) are produced
by the reference plan itself (create-plan + exec); ragged shapes, where the
reference plan is known to write wrong elements, are produced by the
reference's naive transpose RefTrans (test/inc/hptt/test_util.tcc:143-185),
which always reads B and so is used only with beta != 0.
The fixtures pin the oracle restatement on any machine, without the reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")

# (dtype, in_size, perm, alpha, beta)
PLAN_CASES = [
    ("f32", [64, 64], [1, 0], 2.3, 4.2),
    ("f32", [64, 64], [1, 0], 1.0, 0.0),
    ("f32", [16, 16, 16], [2, 1, 0], 2.3, 4.2),
    ("f32", [8, 8, 8, 16], [3, 1, 0, 2], 2.3, 4.2),
    ("f32", [8, 8, 8, 8, 8], [4, 2, 0, 1, 3], 1.0, 0.0),
    ("f64", [4, 8, 4, 4, 8], [1, 0, 2, 4, 3], 2.3, 4.2),
    ("f64", [8, 8, 12, 8], [3, 1, 0, 2], 2.3, 4.2),
    ("f64", [4, 8, 4, 4, 4, 4], [5, 2, 0, 4, 1, 3], 1.0, 0.0),
    ("f64", [8, 8, 4, 8], [0, 3, 2, 1], 2.3, 4.2),
    ("c64", [16, 8, 16], [2, 1, 0], 2.3, 4.2),
    ("c64", [8, 4, 4, 4, 4, 4], [5, 2, 0, 4, 1, 3], 1.5, -0.5),
    ("c128", [16, 8, 16], [2, 1, 0], 2.3, 4.2),
    ("c128", [2, 4, 4, 4, 2, 4], [0, 3, 2, 1, 4, 5], 0.25, 1.0),
]
NAIVE_CASES = [
    ("f32", [13, 11], [1, 0], 2.3, 4.2),
    ("f32", [17, 13, 11], [2, 1, 0], 2.3, 4.2),
    ("f32", [17, 13, 11], [0, 2, 1], 2.3, 4.2),
    ("f64", [10, 7, 9, 5], [3, 1, 0, 2], 2.3, 4.2),
    ("f32", [6, 5, 4, 3, 7], [4, 2, 0, 1, 3], 2.3, 4.2),
    ("c64", [17, 9, 13], [2, 1, 0], 2.3, 4.2),
    ("c128", [3, 5, 2, 3, 2, 3], [5, 4, 3, 2, 1, 0], -1.25, 0.5),
]


def rand(rng, n, name):
    dt = oracle.NP_DTYPES[name]
    x = oracle.aligned_empty(n, dt)
    if name.startswith("c"):
        x[:] = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    else:
        x[:] = rng.uniform(-1, 1, n)
    return x


def main():
    if not oracle.ref_available():
        sys.exit("build the reference first: make -C oracle ref")
    rng = np.random.default_rng(20240601)
    data = {}
    idx = 0
    for source, cases in (("plan", PLAN_CASES), ("naive", NAIVE_CASES)):
        for name, size, perm, al, be in cases:
            n = int(np.prod(size))
            a = rand(rng, n, name)
            b0 = rand(rng, n, name)
            b = oracle.aligned_empty(n, a.dtype)
            b[:] = b0
            if source == "plan":
                assert oracle.ref_plan_is_safe(name, size, perm, be)
                oracle.ref_plan_exec(a, b, size, perm, al, be, threads=1)
            else:
                assert be != 0.0
                oracle.ref_naive_exec(a, b, size, perm, al, be, threads=1)
            key = f"c{idx:02d}"
            data[key + "_meta"] = np.array(
                [oracle.DTYPES[name], len(size)] + list(size) + list(perm), dtype=np.int64)
            data[key + "_scal"] = np.array([al, be], dtype=np.float64)
            data[key + "_src"] = np.array([0 if source == "plan" else 1], dtype=np.int64)
            data[key + "_a"] = np.array(a)
            data[key + "_b0"] = np.array(b0)
            data[key + "_b1"] = np.array(b)
            idx += 1
    np.savez_compressed(OUT, **data)
    print(f"wrote {idx} cases to {OUT} ({os.path.getsize(OUT)} bytes)")


def load(path: str = OUT):
    """Yield dicts: dtype, in_size, perm, alpha, beta, source, a, b0, b1."""
    z = np.load(path)
    names = {v: k for k, v in oracle.DTYPES.items()}
    keys = sorted({k.split("_")[0] for k in z.files})
    for k in keys:
        meta = z[k + "_meta"]
        rank = int(meta[1])
        yield {
            "key": k,
            "dtype": names[int(meta[0])],
            "in_size": [int(x) for x in meta[2:2 + rank]],
            "perm": [int(x) for x in meta[2 + rank:2 + 2 * rank]],
            "alpha": float(z[k + "_scal"][0]),
            "beta": float(z[k + "_scal"][1]),
            "source": "plan" if int(z[k + "_src"][0]) == 0 else "naive",
            "a": z[k + "_a"], "b0": z[k + "_b0"], "b1": z[k + "_b1"],
        }


if __name__ == "__main__":
    main()
