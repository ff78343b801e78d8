"""CPU checkers for the transpose B = alpha * A(perm) + beta * B.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py -- never by the product package ``hptt_b200``.

* ``transpose``      -- the C restatement (oracle/oracle.c -> liboracle.so).
* ``ref_plan_exec``  -- the reference's own CPU plan compiled from its sources
                        (oracle/Makefile -> oracle/_ref/libhptt_ref.so).
* ``ref_naive_exec`` -- the reference's naive OpenMP transpose RefTrans
                        (test/inc/hptt/test_util.tcc:143-185), same library.

The restatement is pinned bit-for-bit against ``ref_plan_exec`` on the shapes
where the reference plan is correct, and against tests/golden/ fixtures that
``ref_plan_exec`` produced.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhptt_ref.so")

DTYPES = {"f32": 0, "f64": 1, "c64": 2, "c128": 3}
NP_DTYPES = {"f32": np.float32, "f64": np.float64, "c64": np.complex64, "c128": np.complex128}

_u32p = ctypes.POINTER(ctypes.c_uint32)
_dp = ctypes.POINTER(ctypes.c_double)


def ref_dir() -> str | None:
    """The reference checkout named by HPTT_REF_DIR, when its sources exist."""
    d = os.environ.get("HPTT_REF_DIR", "")
    return d if d and os.path.isdir(os.path.join(d, "src")) else None


def build(with_ref: bool | None = None) -> None:
    """Compile liboracle.so, and the reference library from the checkout that
    HPTT_REF_DIR names (with_ref None: when that checkout exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if with_ref is None:
        with_ref = ref_dir() is not None
    if with_ref:
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={ref_dir() or ''}"],
                       check=True)


_oracle = None
_ref = None


def _load_oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        lib = ctypes.CDLL(ORACLE_SO)
        lib.hptt_oracle_trans.restype = ctypes.c_int
        lib.hptt_oracle_trans.argtypes = [
            ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, _u32p, _dp, _dp,
            ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        lib.hptt_oracle_update.restype = ctypes.c_int
        lib.hptt_oracle_update.argtypes = [ctypes.c_int, _dp, ctypes.c_int]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _load_ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("reference CPU library not built: " + REF_SO)
        lib = ctypes.CDLL(REF_SO)
        lib.hptt_ref_plan_exec.restype = ctypes.c_int
        lib.hptt_ref_plan_exec.argtypes = [
            ctypes.c_int, ctypes.c_int, _u32p, _u32p, ctypes.c_double,
            ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
            ctypes.c_double, ctypes.c_int, _dp]
        lib.hptt_ref_naive_exec.restype = ctypes.c_int
        lib.hptt_ref_naive_exec.argtypes = [
            ctypes.c_int, ctypes.c_int, _u32p, _u32p, ctypes.c_double,
            ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
            ctypes.c_int, _dp]
        lib.hptt_ref_max_threads.restype = ctypes.c_int
        _ref = lib
    return _ref


def _u32(v):
    arr = (ctypes.c_uint32 * len(v))(*[int(x) for x in v])
    return arr


def _scalar(x):
    z = complex(x)
    return (ctypes.c_double * 2)(z.real, z.imag)


def dtype_name(arr: np.ndarray) -> str:
    for k, v in NP_DTYPES.items():
        if arr.dtype == v:
            return k
    raise TypeError(f"unsupported dtype {arr.dtype}")


def transpose(a: np.ndarray, b: np.ndarray, in_size, perm, alpha, beta,
              in_outer=None, out_outer=None, complex_scalars=None,
              threads: int = 0) -> np.ndarray:
    """Run the restatement in place on flat column-major buffers ``a``/``b``."""
    lib = _load_oracle()
    name = dtype_name(a)
    assert b.dtype == a.dtype and a.flags.c_contiguous and b.flags.c_contiguous
    if complex_scalars is None:
        complex_scalars = name in ("c64", "c128") and (
            complex(alpha).imag != 0 or complex(beta).imag != 0)
    rank = len(in_size)
    rc = lib.hptt_oracle_trans(
        DTYPES[name], rank, _u32(in_size), _u32(perm),
        _u32(in_outer) if in_outer is not None else None,
        _u32(out_outer) if out_outer is not None else None,
        _scalar(alpha), _scalar(beta), int(bool(complex_scalars)),
        a.ctypes.data, b.ctypes.data, int(threads or os.cpu_count() or 1))
    if rc != 0:
        raise ValueError("oracle rejected arguments")
    return b


def updates(name: str, beta, complex_scalars: bool = False) -> bool:
    return bool(_load_oracle().hptt_oracle_update(DTYPES[name], _scalar(beta),
                                                  int(complex_scalars)))


def ref_plan_exec(a: np.ndarray, b: np.ndarray, in_size, perm, alpha: float,
                  beta: float, threads: int = 1, tuning_timeout: float = 0.0,
                  repeat: int = 1) -> float:
    """Run the reference plan in place; returns the best exec time (s)."""
    lib = _load_ref()
    name = dtype_name(a)
    best = ctypes.c_double(0.0)
    rc = lib.hptt_ref_plan_exec(DTYPES[name], len(in_size), _u32(in_size),
                                _u32(perm), float(alpha), float(beta),
                                a.ctypes.data, b.ctypes.data, int(threads),
                                float(tuning_timeout), int(repeat),
                                ctypes.byref(best))
    if rc != 0:
        raise ValueError("reference plan rejected arguments")
    return best.value


def ref_naive_exec(a: np.ndarray, b: np.ndarray, in_size, perm, alpha: float,
                   beta: float, threads: int = 1, repeat: int = 1) -> float:
    lib = _load_ref()
    name = dtype_name(a)
    best = ctypes.c_double(0.0)
    rc = lib.hptt_ref_naive_exec(DTYPES[name], len(in_size), _u32(in_size),
                                 _u32(perm), float(alpha), float(beta),
                                 a.ctypes.data, b.ctypes.data, int(threads),
                                 int(repeat), ctypes.byref(best))
    if rc != 0:
        raise ValueError("reference naive transpose rejected arguments")
    return best.value


def ref_plan_is_safe(name: str, in_size, perm, beta: float) -> bool:
    """Shapes on which the reference plan is known to be correct.

    The reference's ragged-edge kernel writes through the input offset
    (src/kernels/macro_kernel_trans.cc:236,248) and its beta == 0 streaming
    stores assume aligned rows and mis-step on complex types
    (macro_kernel_trans.cc:60-77, inc/hptt/arch/avx2/kernel_trans_avx2.tcc:35-37).
    It is exact when every extent is a multiple of the vector width (32 bytes
    / element size) and, for complex types, beta != 0.
    """
    width = {"f32": 8, "f64": 4, "c64": 4, "c128": 2}[name]
    if any(int(n) % width for n in in_size):
        return False
    if name in ("c64", "c128") and abs(beta) < 1e-16:
        return False
    return True


def aligned_empty(n: int, dtype, align: int = 4096) -> np.ndarray:
    """Page-aligned 1-D array (the reference's vector kernels use aligned loads)."""
    itemsize = np.dtype(dtype).itemsize
    raw = np.empty(n * itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * itemsize].view(dtype)
