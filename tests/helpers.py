"""Shared helpers for the parity tests: seeded inputs, GPU runs through the
C ABI, and bit-level comparison against the oracle."""
from __future__ import annotations

import numpy as np

import oracle

NP = oracle.NP_DTYPES
REAL_OF = {"f32": np.float32, "f64": np.float64, "c64": np.float32, "c128": np.float64}
UINT_OF = {"f32": np.uint32, "f64": np.uint64, "c64": np.uint32, "c128": np.uint64}


def footprint(in_size, perm, in_outer=None, out_outer=None):
    n_in = int(np.prod(in_outer if in_outer is not None else in_size))
    out_size = [in_size[p] for p in perm]
    n_out = int(np.prod(out_outer if out_outer is not None else out_size))
    return n_in, n_out


def seeded(rng, n, name, lo=-1.0, hi=1.0):
    dt = NP[name]
    x = oracle.aligned_empty(n, dt)
    if name in ("c64", "c128"):
        x[:] = rng.uniform(lo, hi, n) + 1j * rng.uniform(lo, hi, n)
    else:
        x[:] = rng.uniform(lo, hi, n)
    return x


def as_real_view(x: np.ndarray, name: str) -> np.ndarray:
    return x.view(REAL_OF[name])


def assert_same(got: np.ndarray, want: np.ndarray, name: str, what: str = ""):
    """Bit-exact comparison.  NaN matches NaN (payloads differ between the
    host's x86 multiply and the GPU's canonical NaN)."""
    g = as_real_view(got, name)
    w = as_real_view(want, name)
    gb = g.view(UINT_OF[name])
    wb = w.view(UINT_OF[name])
    same = gb == wb
    both_nan = np.isnan(g) & np.isnan(w)
    bad = ~(same | both_nan)
    if bad.any():
        idx = np.flatnonzero(bad)
        i = int(idx[0])
        raise AssertionError(
            f"{what}: {idx.size} of {bad.size} components differ; first at {i}: "
            f"got {g[i]!r} want {w[i]!r}")


def oracle_run(name, in_size, perm, alpha, beta, a, b0, in_outer=None, out_outer=None,
               complex_scalars=None):
    want = oracle.aligned_empty(b0.size, b0.dtype)
    want[:] = b0
    oracle.transpose(a, want, in_size, perm, alpha, beta, in_outer=in_outer,
                     out_outer=out_outer, complex_scalars=complex_scalars)
    return want


def gpu_run(name, in_size, perm, alpha, beta, a, b0, in_outer=None, out_outer=None,
            complex_scalars=None, tuning_timeout=0.0, device_offset_bytes=0):
    """Run one transpose through the C ABI on cuda:0; returns B on the host."""
    import torch
    import hptt_b200 as h
    tdt = {"f32": torch.float32, "f64": torch.float64, "c64": torch.complex64,
           "c128": torch.complex128}[name]
    esz = np.dtype(NP[name]).itemsize
    assert device_offset_bytes % esz == 0
    off = device_offset_bytes // esz
    da = torch.empty(a.size + off, dtype=tdt, device="cuda")
    db = torch.empty(b0.size + off, dtype=tdt, device="cuda")
    da[off:].copy_(torch.from_numpy(np.asarray(a)))
    db[off:].copy_(torch.from_numpy(np.asarray(b0)))
    ap, bp = da[off:], db[off:]
    plan = h.create_plan(ap, bp, in_size, perm, alpha, beta, 1, tuning_timeout,
                         in_outer or (), out_outer or (), dtype=name,
                         complex_scalars=complex_scalars)
    assert plan is not None
    plan.exec()
    plan.sync()
    out = bp.cpu().numpy()
    plan.destroy()
    return out


def random_perm(rng, rank, non_identity=True):
    while True:
        p = list(rng.permutation(rank))
        if not non_identity or p != list(range(rank)):
            return [int(x) for x in p]
