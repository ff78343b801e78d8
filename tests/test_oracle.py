"""The oracle restatement, pinned against the reference's own CPU code.

* every committed golden fixture (made by the reference plan, or by its naive
  RefTrans on ragged shapes) is reproduced bit-for-bit;
* when the reference library is built in this container, fresh seeded cases
  on the plan's correct subset are compared bit-for-bit as well;
* tiny cases are checked against a pure-Python loop (outer sizes, complex
  scalars, beta below the update threshold).
"""
import itertools

import numpy as np
import pytest

import oracle
from golden.make_golden import load as load_golden
from helpers import assert_same, footprint, oracle_run, seeded


@pytest.mark.parametrize("case", list(load_golden()), ids=lambda c: c["key"])
def test_oracle_matches_reference_golden(case):
    name = case["dtype"]
    a = case["a"]
    want = case["b1"]
    got = oracle_run(name, case["in_size"], case["perm"], case["alpha"], case["beta"],
                     a, case["b0"].copy())
    assert_same(got, want, name, f"golden {case['key']} ({case['source']})")


REF_CASES = [
    ("f32", [256, 256, 256], [2, 1, 0], 2.3, 4.2),   # the plain single-transpose workload
    ("f32", [64, 64], [1, 0], 1.0, 0.0),
    ("f32", [8, 16, 8, 16, 8], [4, 2, 0, 1, 3], 2.3, 4.2),
    ("f32", [16, 8, 8, 16], [0, 3, 2, 1], 1.0, 0.0),
    ("f64", [16, 8, 12, 8], [3, 1, 0, 2], 2.3, 4.2),
    ("f64", [8, 8, 4, 8, 8, 4], [5, 2, 0, 4, 1, 3], 1.0, 0.0),
    ("c64", [16, 8, 16], [2, 1, 0], 2.3, 4.2),
    ("c64", [8, 16, 4, 16, 4, 8], [5, 2, 0, 4, 1, 3], -0.75, 1.5),
    ("c128", [16, 8, 16], [2, 1, 0], 2.3, 4.2),
    ("c128", [8, 4, 4, 8, 2, 4], [0, 3, 2, 1, 4, 5], 2.3, 4.2),
]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("name,size,perm,al,be", REF_CASES)
def test_oracle_matches_reference_plan(name, size, perm, al, be):
    assert oracle.ref_plan_is_safe(name, size, perm, be)
    rng = np.random.default_rng(0)
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    b0 = seeded(rng, n, name)
    ref = oracle.aligned_empty(n, a.dtype)
    ref[:] = b0
    oracle.ref_plan_exec(a, ref, size, perm, al, be, threads=2)
    got = oracle_run(name, size, perm, al, be, a, b0)
    assert_same(got, ref, name, "oracle vs reference plan")


def _py_transpose(name, in_size, perm, alpha, beta, a, b, in_outer=None, out_outer=None,
                  complex_scalars=False):
    """Pure-Python statement of the same arithmetic (small cases only)."""
    rank = len(in_size)
    io = in_outer or in_size
    oo = out_outer or [in_size[p] for p in perm]
    sa = [int(np.prod(io[:d])) for d in range(rank)]
    so = [int(np.prod(oo[:k])) for k in range(rank)]
    real = np.float32 if name in ("f32", "c64") else np.float64
    cplx = name in ("c64", "c128")
    upd = oracle.updates(name, beta, complex_scalars)
    al, be = complex(alpha), complex(beta)
    for idx in itertools.product(*[range(n) for n in in_size]):
        ia = sum(i * s for i, s in zip(idx, sa))
        ib = sum(idx[perm[k]] * so[k] for k in range(rank))
        x = a[ia]
        if not cplx:
            t = real(real(al.real) * real(x))
            if upd:
                t = real(t + real(real(be.real) * real(b[ib])))
            b[ib] = t
            continue
        xr, xi = real(x.real), real(x.imag)
        if complex_scalars:
            tr = real(real(real(al.real) * xr) - real(real(al.imag) * xi))
            ti = real(real(real(al.real) * xi) + real(real(al.imag) * xr))
        else:
            tr, ti = real(real(al.real) * xr), real(real(al.real) * xi)
        if upd:
            yr, yi = real(b[ib].real), real(b[ib].imag)
            if complex_scalars:
                ur = real(real(real(be.real) * yr) - real(real(be.imag) * yi))
                ui = real(real(real(be.real) * yi) + real(real(be.imag) * yr))
            else:
                ur, ui = real(real(be.real) * yr), real(real(be.real) * yi)
            tr, ti = real(tr + ur), real(ti + ui)
        b[ib] = tr + 1j * ti
    return b


SMALL = [
    ("f32", [3, 4], [1, 0], 2.3, 4.2, None, None, False),
    ("f32", [3, 4, 5], [2, 0, 1], 1.0, 0.0, None, None, False),
    ("f64", [2, 3, 2, 3], [3, 1, 0, 2], -0.5, 1e-17, None, None, False),  # beta below threshold
    ("f32", [3, 4, 2], [1, 2, 0], 2.3, 4.2, [5, 4, 3], [6, 2, 4], False),  # outer sizes
    ("c64", [3, 2, 4], [2, 1, 0], 1.5 - 0.5j, 0.25 + 1j, None, None, True),
    ("c128", [2, 3, 2, 2], [0, 3, 2, 1], 1.5 - 0.5j, 0.25 + 1j, [3, 3, 2, 2], None, True),
    ("c128", [2, 3, 3], [1, 2, 0], 2.0, -1.0, None, None, False),
]


@pytest.mark.parametrize("name,size,perm,al,be,io,oo,cs", SMALL)
def test_oracle_matches_python_loop(name, size, perm, al, be, io, oo, cs):
    rng = np.random.default_rng(1)
    n_in, n_out = footprint(size, perm, io, oo)
    a = seeded(rng, n_in, name)
    b0 = seeded(rng, n_out, name)
    got = oracle_run(name, size, perm, al, be, a, b0, io, oo, complex_scalars=cs)
    want = _py_transpose(name, size, perm, al, be, a, b0.copy(), io, oo, complex_scalars=cs)
    assert_same(got, want, name, "oracle vs python loop")


def test_oracle_skips_b_below_threshold():
    """|beta| < 1e-16: B is not read, so NaN in B does not propagate
    (inc/hptt/impl/hptt_trans_impl.h:75-78)."""
    rng = np.random.default_rng(2)
    a = seeded(rng, 12, "f64")
    b0 = np.full(12, np.nan)
    got = oracle_run("f64", [3, 4], [1, 0], 2.0, 5e-17, a, b0)
    assert not np.isnan(got).any()
    got2 = oracle_run("f64", [3, 4], [1, 0], 2.0, 2e-16, a, b0)
    assert np.isnan(got2).all()
