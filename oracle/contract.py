"""CPU checker for tensor contractions run as transpose - GEMM - transpose.

TEST INFRASTRUCTURE ONLY.  Imported by tests/ and bench.py's checks -- never by
the product package ``hptt_b200``.

    C[lc] = alpha * sum_K A[la] * B[lb] + beta * C[lc]

Tensors are flat column-major buffers (stride-1 dimension first), the layout
of the transposes (reference inc/hptt/tensor.tcc:186-196).  C is read only
when |beta| >= 1e-16, the transposes' update rule (reference
inc/hptt/impl/hptt_trans_impl.h:75-78); complex types with real scalars scale
both components (inc/hptt/types.h:29-54).

The reference has no contraction code, so nothing here is pinned to it
beyond those rules: ``contract`` evaluates the sum in extended precision
(numpy longdouble, 64-bit mantissa on x86) and returns with it an elementwise
bound on the rounding error of any summation order in the element type --
the standard dot-product bound |fl(s) - s| <= gamma_K * sum |a| |b| with
gamma_K = K u / (1 - K u), widened for the scalar multiplies, the beta term
and complex arithmetic.
"""
from __future__ import annotations

import string

import numpy as np

EPS = {"f32": np.finfo(np.float32).eps / 2, "f64": np.finfo(np.float64).eps / 2,
       "c64": np.finfo(np.float32).eps / 2, "c128": np.finfo(np.float64).eps / 2}
NP = {"f32": np.float32, "f64": np.float64, "c64": np.complex64, "c128": np.complex128}


def _letters(la, lb, lc):
    codes = {}
    for x in list(la) + list(lb) + list(lc):
        if x not in codes:
            codes[x] = string.ascii_letters[len(codes)]
    return ("".join(codes[x] for x in la), "".join(codes[x] for x in lb),
            "".join(codes[x] for x in lc))


def beta_reads(name, beta, complex_scalars=False):
    if complex_scalars:
        return abs(complex(beta).real) >= 1e-16 or abs(complex(beta).imag) >= 1e-16
    b = float(complex(beta).real)
    if name in ("f32", "c64"):
        b = float(np.float32(b))
    return abs(b) >= 1e-16


def out_size(size_a, la, size_b, lb, lc):
    ext = dict(zip(la, size_a))
    ext.update(zip(lb, size_b))
    return [int(ext[x]) for x in lc]


def contract(name, size_a, la, a, size_b, lb, b, lc, c0, alpha, beta, complex_scalars=False):
    """Returns (value, bound): the exact-ish result in extended precision and
    the per-element error allowance, both flat in C's column-major order."""
    sa, sb, sc = _letters(la, lb, lc)
    cplx = name in ("c64", "c128")
    ext_t = np.clongdouble if cplx else np.longdouble
    A = np.asarray(a).reshape(list(size_a), order="F").astype(ext_t)
    B = np.asarray(b).reshape(list(size_b), order="F").astype(ext_t)
    prod = np.einsum(f"{sa},{sb}->{sc}", A, B)
    absprod = np.einsum(f"{sa},{sb}->{sc}", np.abs(A).astype(np.longdouble),
                        np.abs(B).astype(np.longdouble))
    if cplx and complex_scalars:
        al, be = complex(alpha), complex(beta)
    elif cplx:
        al, be = complex(complex(alpha).real, 0), complex(complex(beta).real, 0)
    else:
        al, be = float(complex(alpha).real), float(complex(beta).real)
    if name in ("f32", "c64"):  # scalars enter the device in the element precision
        al = complex(np.float32(complex(al).real), np.float32(complex(al).imag)) if cplx \
            else float(np.float32(al))
        be = complex(np.float32(complex(be).real), np.float32(complex(be).imag)) if cplx \
            else float(np.float32(be))
    ext_al = ext_t(al)
    val = ext_al * prod
    bnd_terms = abs(al) * absprod
    if beta_reads(name, beta, complex_scalars):
        C0 = np.asarray(c0).reshape(list(out_size(size_a, la, size_b, lb, lc)),
                                    order="F").astype(ext_t)
        val = val + ext_t(be) * C0
        bnd_terms = bnd_terms + abs(be) * np.abs(C0).astype(np.longdouble)
    k = 1
    ext = dict(zip(la, size_a))
    for x in la:
        if x in lb and x not in lc:
            k *= int(ext[x])
    u = EPS[name]
    gamma = (k + 6) * u / (1 - (k + 6) * u) * (4.0 if cplx else 1.0)
    # the smallest normal of the type covers underflow of tiny products
    tiny = np.finfo(np.float32 if name in ("f32", "c64") else np.float64).tiny
    bound = gamma * bnd_terms + tiny * (k + 2)
    return (np.asarray(val).reshape(-1, order="F"), np.asarray(bound).reshape(-1, order="F"))


def check(name, got, value, bound, what=""):
    """Assert |got - value| <= bound elementwise (complex: componentwise)."""
    got = np.asarray(got)
    if name in ("c64", "c128"):
        err = np.maximum(np.abs(got.real.astype(np.longdouble) - value.real),
                         np.abs(got.imag.astype(np.longdouble) - value.imag))
    else:
        err = np.abs(got.astype(np.longdouble) - value)
    bad = ~(err <= bound)
    if bad.any():
        i = int(np.flatnonzero(bad)[0])
        raise AssertionError(
            f"{what}: {int(bad.sum())} of {bad.size} elements beyond the error bound; first "
            f"at {i}: got {got[i]!r} want {value[i]!r} err {err[i]!r} bound {bound[i]!r}")
