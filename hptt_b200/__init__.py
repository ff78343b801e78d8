"""hptt_b200 -- B200 (sm_100a) tensor transposition B = alpha * A(perm) + beta * B.

Python mirror of the reference's plan interface, bound to the C ABI of
``libhptt_cuda.so`` (include/hptt_cuda.h) with ctypes:

    plan = hptt_b200.create_plan(a, b, in_size, perm, alpha, beta, num_threads)
    if plan is not None:
        plan.exec()

``create_plan`` mirrors ``hptt::create_plan`` (reference inc/hptt/hptt.h:85-93):
same argument meaning and order, and ``None`` where the reference returns
``nullptr`` (invalid arguments, inc/hptt/hptt.h:71-83).  The plan object has the
reference's methods ``exec``, ``__call__``, ``print_plan``, ``reset_data``,
``set_thread_ids`` and ``unset_thread_ids`` (inc/hptt/impl/hptt_trans.h:26-31),
plus ``sync`` and ``set_stream`` because ``exec`` is asynchronous on the GPU.

Data are device buffers: torch CUDA tensors, objects exposing
``__cuda_array_interface__``, or raw device addresses (int).  Tensors are flat
column-major buffers: dimension 0 has stride 1.

There is no CPU fallback: importing works anywhere, but creating a plan needs
the compiled library and a CUDA device, and raises if either is missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhptt_cuda.so")

F32, F64, C64, C128 = 0, 1, 2, 3
_DTYPE_NAMES = {"f32": F32, "float32": F32, "float": F32,
                "f64": F64, "float64": F64, "double": F64,
                "c64": C64, "complex64": C64, "cfloat": C64,
                "c128": C128, "complex128": C128, "cdouble": C128}
ELEM_BYTES = {F32: 4, F64: 8, C64: 8, C128: 16}

STATUS = {
    0: "ok", 1: "null data pointer", 2: "bad rank", 3: "bad size vector",
    4: "bad size value", 5: "bad permutation", 6: "bad dtype", 7: "CUDA error",
    8: "no CUDA device", 9: "allocation failed", 10: "memory budget exceeded",
    11: "invalid handle", 12: "timeout", 13: "too large", 14: "busy",
    15: "labels do not describe a contraction", 16: "cuBLAS error",
}
# argument errors for which the reference returns nullptr
_NULLPTR_STATUSES = {1, 2, 3, 4, 5}


class HpttError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")


_lib = None
_u32p = ctypes.POINTER(ctypes.c_uint32)
_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)


def library_path() -> str:
    return LIB_PATH


class ServeConfig(ctypes.Structure):
    """hptt_cuda_serve_config"""
    _fields_ = [("budget_bytes", ctypes.c_uint64), ("max_inflight_launches", ctypes.c_uint32),
                ("max_batch", ctypes.c_uint32), ("per_call", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class ServeStats(ctypes.Structure):
    """hptt_cuda_serve_stats"""
    _fields_ = [(n, ctypes.c_uint64) for n in (
                    "submitted", "completed", "failed", "launches", "bytes",
                    "peak_inflight_bytes", "peak_pending")] + \
               [(n, ctypes.c_double) for n in (
                    "elapsed_s", "throughput_rps", "gbs", "mean_batch", "lat_mean_us",
                    "lat_p50_us", "lat_p99_us", "lat_p999_us", "lat_max_us",
                    "sched_pass_max_us")]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class ContractStats(ctypes.Structure):
    """hptt_cuda_contract_stats (include/hptt_cuda.h)."""
    _fields_ = [("m", ctypes.c_uint64), ("n", ctypes.c_uint64), ("k", ctypes.c_uint64),
                ("batch", ctypes.c_uint64), ("flops", ctypes.c_uint64),
                ("transpose_bytes", ctypes.c_uint64), ("workspace_bytes", ctypes.c_uint64),
                ("transposes", ctypes.c_uint32), ("graph", ctypes.c_uint32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def load_library() -> ctypes.CDLL:
    """Load libhptt_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m hptt_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    c_int, c_u32, c_vp, c_dbl, c_sz = (ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p,
                                       ctypes.c_double, ctypes.c_size_t)
    sigs = {
        "hptt_cuda_plan_create": (c_int, [c_int, c_u32, _u32p, _u32p, _u32p, _u32p, _dp, _dp,
                                          c_int, c_vp, c_vp, c_u32, c_dbl,
                                          ctypes.POINTER(c_vp)]),
        "hptt_cuda_plan_exec": (c_int, [c_vp]),
        "hptt_cuda_plan_exec_on": (c_int, [c_vp, c_vp]),
        "hptt_cuda_plan_reset_data": (c_int, [c_vp, c_vp, c_vp]),
        "hptt_cuda_plan_describe": (c_int, [c_vp, ctypes.c_char_p, c_sz]),
        "hptt_cuda_plan_set_thread_ids": (c_int, [c_vp, ctypes.POINTER(ctypes.c_int32), c_u32]),
        "hptt_cuda_plan_unset_thread_ids": (c_int, [c_vp]),
        "hptt_cuda_plan_set_stream": (c_int, [c_vp, c_vp]),
        "hptt_cuda_plan_sync": (c_int, [c_vp]),
        "hptt_cuda_plan_set_coef": (c_int, [c_vp, _dp, _dp, c_int]),
        "hptt_cuda_plan_bytes": (c_int, [c_vp, ctypes.POINTER(ctypes.c_uint64)]),
        "hptt_cuda_plan_launches": (c_int, [c_vp, ctypes.POINTER(c_u32)]),
        "hptt_cuda_plan_destroy": (c_int, [c_vp]),
        "hptt_cuda_plan_inspect": (c_int, [c_int, c_u32, _u32p, _u32p, _u32p, _u32p,
                                           ctypes.c_char_p, c_sz]),
        "hptt_cuda_batch_create": (c_int, [ctypes.POINTER(c_vp), c_u32, ctypes.POINTER(c_vp)]),
        "hptt_cuda_batch_refresh": (c_int, [c_vp]),
        "hptt_cuda_batch_exec": (c_int, [c_vp, c_vp]),
        "hptt_cuda_batch_info": (c_int, [c_vp, ctypes.POINTER(ctypes.c_uint64),
                                         ctypes.POINTER(c_u32), ctypes.POINTER(c_u32)]),
        "hptt_cuda_batch_destroy": (c_int, [c_vp]),
        "hptt_cuda_plan_exec_many": (c_int, [ctypes.POINTER(c_vp), c_u32, c_vp]),
        "hptt_cuda_server_create": (c_int, [ctypes.POINTER(ServeConfig), ctypes.POINTER(c_vp)]),
        "hptt_cuda_server_submit": (c_int, [c_vp, c_vp, c_vp, c_vp,
                                            ctypes.POINTER(ctypes.c_uint64)]),
        "hptt_cuda_server_wait": (c_int, [c_vp, ctypes.c_uint64, c_dbl]),
        "hptt_cuda_server_drain": (c_int, [c_vp, c_dbl]),
        "hptt_cuda_server_stats": (c_int, [c_vp, ctypes.POINTER(ServeStats)]),
        "hptt_cuda_server_reset_stats": (c_int, [c_vp]),
        "hptt_cuda_server_run_poisson": (c_int, [c_vp, ctypes.POINTER(c_vp), c_u32, c_dbl, c_dbl,
                                                 ctypes.c_uint64, c_dbl,
                                                 ctypes.POINTER(ServeStats)]),
        "hptt_cuda_server_destroy": (c_int, [c_vp]),
        "hptt_cuda_contract_create": (c_int, [c_int, c_u32, _u32p, _i32p, c_u32, _u32p, _i32p,
                                              c_u32, _i32p, _dp, _dp, c_int, c_vp, c_vp, c_vp,
                                              c_vp, ctypes.c_uint64, ctypes.POINTER(c_vp)]),
        "hptt_cuda_contract_inspect": (c_int, [c_int, c_u32, _u32p, _i32p, c_u32, _u32p, _i32p,
                                               c_u32, _i32p, ctypes.c_char_p, c_sz,
                                               ctypes.POINTER(ctypes.c_uint64)]),
        "hptt_cuda_contract_exec": (c_int, [c_vp]),
        "hptt_cuda_contract_exec_on": (c_int, [c_vp, c_vp]),
        "hptt_cuda_contract_reset_data": (c_int, [c_vp, c_vp, c_vp, c_vp]),
        "hptt_cuda_contract_set_coef": (c_int, [c_vp, _dp, _dp, c_int]),
        "hptt_cuda_contract_set_stream": (c_int, [c_vp, c_vp]),
        "hptt_cuda_contract_set_graph": (c_int, [c_vp, c_int]),
        "hptt_cuda_contract_sync": (c_int, [c_vp]),
        "hptt_cuda_contract_info": (c_int, [c_vp, ctypes.POINTER(ContractStats)]),
        "hptt_cuda_contract_describe": (c_int, [c_vp, ctypes.c_char_p, c_sz]),
        "hptt_cuda_contract_destroy": (c_int, [c_vp]),
        "hptt_cuda_tune_cache_load": (c_int, [ctypes.c_char_p]),
        "hptt_cuda_tune_cache_save": (c_int, [ctypes.c_char_p]),
        "hptt_cuda_tune_cache_clear": (c_int, []),
        "hptt_cuda_tune_cache_size": (c_int, [ctypes.POINTER(c_u32)]),
        "hptt_cuda_status_string": (ctypes.c_char_p, [c_int]),
        "hptt_cuda_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _u32(v: Optional[Sequence[int]]):
    if v is None:
        return None
    return (ctypes.c_uint32 * len(v))(*[int(x) for x in v])


def _scalar(x) -> ctypes.Array:
    z = complex(x)
    return (ctypes.c_double * 2)(z.real, z.imag)


def _device_ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    iface = getattr(x, "__cuda_array_interface__", None)
    if iface is not None:
        return int(iface["data"][0])
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    raise TypeError(f"cannot take a device address of {type(x)!r}")


def dtype_code(x) -> int:
    """Element type code from a name, a torch dtype/tensor or a numpy dtype."""
    if isinstance(x, int):
        return x
    if isinstance(x, str):
        return _DTYPE_NAMES[x]
    dt = getattr(x, "dtype", x)
    name = str(dt).replace("torch.", "")
    if name in _DTYPE_NAMES:
        return _DTYPE_NAMES[name]
    raise TypeError(f"unsupported element type {dt!r}")


class TransPlan:
    """A transpose plan bound to device buffers (reference ``trans_plan<T>``)."""

    def __init__(self, handle: int, dtype: int, keep=()):
        self._h = ctypes.c_void_p(handle)
        self.dtype = dtype
        self._keep = list(keep)  # keep tensors alive while the plan holds them

    # -- reference interface (inc/hptt/impl/hptt_trans.h:26-31) --
    def exec(self) -> None:
        self._check(load_library().hptt_cuda_plan_exec(self._h), "exec")

    def __call__(self) -> None:
        self.exec()

    def print_plan(self) -> None:
        print(self.describe(), end="")

    def reset_data(self, in_data, out_data) -> None:
        self._check(load_library().hptt_cuda_plan_reset_data(
            self._h, _device_ptr(in_data), _device_ptr(out_data)), "reset_data")
        self._keep = [in_data, out_data]

    def set_thread_ids(self, thread_ids: Sequence[int]) -> None:
        arr = (ctypes.c_int32 * len(thread_ids))(*thread_ids)
        self._check(load_library().hptt_cuda_plan_set_thread_ids(self._h, arr, len(thread_ids)),
                    "set_thread_ids")

    def unset_thread_ids(self) -> None:
        self._check(load_library().hptt_cuda_plan_unset_thread_ids(self._h), "unset_thread_ids")

    # -- extensions --
    def exec_on(self, stream) -> None:
        self._check(load_library().hptt_cuda_plan_exec_on(self._h, _stream_ptr(stream)),
                    "exec_on")

    def set_stream(self, stream) -> None:
        self._check(load_library().hptt_cuda_plan_set_stream(self._h, _stream_ptr(stream)),
                    "set_stream")

    def sync(self) -> None:
        self._check(load_library().hptt_cuda_plan_sync(self._h), "sync")

    def set_coef(self, alpha, beta, complex_scalars: bool = False) -> None:
        self._check(load_library().hptt_cuda_plan_set_coef(
            self._h, _scalar(alpha), _scalar(beta), int(complex_scalars)), "set_coef")

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(4096)
        self._check(load_library().hptt_cuda_plan_describe(self._h, buf, 4096), "describe")
        return buf.value.decode()

    @property
    def bytes(self) -> int:
        v = ctypes.c_uint64(0)
        self._check(load_library().hptt_cuda_plan_bytes(self._h, ctypes.byref(v)), "bytes")
        return int(v.value)

    @property
    def launches(self) -> int:
        v = ctypes.c_uint32(0)
        self._check(load_library().hptt_cuda_plan_launches(self._h, ctypes.byref(v)), "launches")
        return int(v.value)

    @property
    def handle(self) -> int:
        return int(self._h.value or 0)

    def destroy(self) -> None:
        if self._h and self._h.value:
            load_library().hptt_cuda_plan_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @staticmethod
    def _check(st: int, what: str) -> None:
        if st != 0:
            raise HpttError(st, what)


def _stream_ptr(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return int(getattr(stream, "cuda_stream"))


def create_plan(in_data, out_data, in_size: Sequence[int], perm: Sequence[int],
                alpha, beta, num_threads: int = 0, tuning_timeout: float = 0.0,
                in_outer_size: Sequence[int] = (), out_outer_size: Sequence[int] = (),
                dtype=None, complex_scalars: Optional[bool] = None) -> Optional[TransPlan]:
    """Mirror of ``hptt::create_plan`` (reference inc/hptt/hptt.h:85-93).

    Returns ``None`` exactly where the reference returns ``nullptr``: a null
    data pointer, rank < 2, a size vector of the wrong length, a zero extent or
    an outer size below the inner size, or an invalid permutation.  Device or
    library failures raise :class:`HpttError`.

    ``alpha``/``beta`` are real scalars as in the reference; for complex
    element types a Python complex (or ``complex_scalars=True``) selects the
    complex-scalar extension.
    """
    code = dtype_code(dtype if dtype is not None else in_data)
    rank = len(perm)
    if rank <= 1:
        return None
    if len(in_size) != rank:
        return None
    if (len(in_outer_size) not in (0, rank)) or (len(out_outer_size) not in (0, rank)):
        return None
    ip, op = _device_ptr(in_data), _device_ptr(out_data)
    if complex_scalars is None:
        complex_scalars = code in (C64, C128) and (
            isinstance(alpha, complex) or isinstance(beta, complex))
    lib = load_library()
    h = ctypes.c_void_p(0)
    st = lib.hptt_cuda_plan_create(
        code, rank, _u32(in_size), _u32(perm),
        _u32(in_outer_size) if len(in_outer_size) else None,
        _u32(out_outer_size) if len(out_outer_size) else None,
        _scalar(alpha), _scalar(beta), int(bool(complex_scalars)),
        ip, op, int(num_threads), float(tuning_timeout), ctypes.byref(h))
    if st in _NULLPTR_STATUSES:
        return None
    if st != 0:
        raise HpttError(st, "create_plan")
    return TransPlan(h.value, code, keep=(in_data, out_data))


def inspect_plan(dtype, in_size: Sequence[int], perm: Sequence[int],
                 in_outer_size: Sequence[int] = (), out_outer_size: Sequence[int] = ()) -> str:
    """Host-only dry run of the planner (no device, no data)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(4096)
    st = lib.hptt_cuda_plan_inspect(
        dtype_code(dtype), len(perm), _u32(in_size), _u32(perm),
        _u32(in_outer_size) if len(in_outer_size) else None,
        _u32(out_outer_size) if len(out_outer_size) else None, buf, 4096)
    if st != 0:
        raise HpttError(st, "inspect_plan")
    return buf.value.decode()


def _handles(plans) -> ctypes.Array:
    arr = (ctypes.c_void_p * max(1, len(plans)))()
    for i, p in enumerate(plans):
        arr[i] = p.handle if p is not None else None
    return arr


class TransBatch:
    """Many plans run by one graph launch (hptt_cuda_batch_*).  Results are
    bit-identical to each plan's own exec.  The plans must stay alive (the
    batch keeps references) and must not write into one another's buffers."""

    def __init__(self, plans: Sequence["TransPlan"]):
        self._plans = list(plans)
        h = ctypes.c_void_p(0)
        st = load_library().hptt_cuda_batch_create(_handles(self._plans), len(self._plans),
                                                   ctypes.byref(h))
        if st != 0:
            raise HpttError(st, "batch_create")
        self._h = h.value

    def exec(self, stream=None) -> None:
        """Enqueue one run of every entry (one graph launch)."""
        st = load_library().hptt_cuda_batch_exec(self._h, _stream_ptr(stream))
        if st != 0:
            raise HpttError(st, "batch_exec")

    def refresh(self) -> None:
        """Re-read the plans' pointers and scalars (after reset_data / set_coef)."""
        st = load_library().hptt_cuda_batch_refresh(self._h)
        if st != 0:
            raise HpttError(st, "batch_refresh")

    def info(self):
        """(algorithmic bytes per exec, work items, kernels per exec)."""
        b, w, k = ctypes.c_uint64(0), ctypes.c_uint32(0), ctypes.c_uint32(0)
        st = load_library().hptt_cuda_batch_info(self._h, ctypes.byref(b), ctypes.byref(w),
                                                 ctypes.byref(k))
        if st != 0:
            raise HpttError(st, "batch_info")
        return int(b.value), int(w.value), int(k.value)

    @property
    def bytes(self) -> int:
        return self.info()[0]

    def destroy(self) -> None:
        if getattr(self, "_h", None):
            load_library().hptt_cuda_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def create_batch(plans: Sequence["TransPlan"]) -> TransBatch:
    return TransBatch(plans)


def exec_many(plans: Sequence["TransPlan"], stream=None) -> None:
    """One plain exec per plan, in order, from a C loop (the per-call form)."""
    st = load_library().hptt_cuda_plan_exec_many(_handles(plans), len(plans),
                                                 _stream_ptr(stream))
    if st != 0:
        raise HpttError(st, "exec_many")


class TransServer:
    """The served form (hptt_cuda_server_*): requests are queued, admitted
    against a device-byte budget and run with continuous batching (or one
    plain exec each with ``per_call=True``).  Buffers passed to ``submit``
    must stay alive until the request has finished."""

    def __init__(self, budget_bytes: int = 32 << 30, max_inflight_launches: int = 4,
                 max_batch: int = 512, per_call: bool = False):
        cfg = ServeConfig(int(budget_bytes), int(max_inflight_launches), int(max_batch),
                          int(bool(per_call)), 0)
        h = ctypes.c_void_p(0)
        st = load_library().hptt_cuda_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise HpttError(st, "server_create")
        self._h = h.value

    def submit(self, plan: "TransPlan", in_data=None, out_data=None) -> int:
        t = ctypes.c_uint64(0)
        ip = _device_ptr(in_data) if in_data is not None else None
        op = _device_ptr(out_data) if out_data is not None else None
        st = load_library().hptt_cuda_server_submit(self._h, plan.handle, ip, op,
                                                    ctypes.byref(t))
        if st != 0:
            raise HpttError(st, "server_submit")
        return int(t.value)

    def wait(self, ticket: int, timeout: float = 60.0) -> None:
        st = load_library().hptt_cuda_server_wait(self._h, ticket, float(timeout))
        if st != 0:
            raise HpttError(st, f"server_wait({ticket})")

    def drain(self, timeout: float = 120.0) -> None:
        st = load_library().hptt_cuda_server_drain(self._h, float(timeout))
        if st != 0:
            raise HpttError(st, "server_drain")

    def stats(self) -> dict:
        s = ServeStats()
        st = load_library().hptt_cuda_server_stats(self._h, ctypes.byref(s))
        if st != 0:
            raise HpttError(st, "server_stats")
        return s.as_dict()

    def reset_stats(self) -> None:
        st = load_library().hptt_cuda_server_reset_stats(self._h)
        if st != 0:
            raise HpttError(st, "server_reset_stats")

    def run_poisson(self, pool: Sequence["TransPlan"], rate: float, seconds: float,
                    seed: int = 0, drain_timeout: float = 300.0) -> dict:
        """Open-loop Poisson arrivals over `pool` (native load generator)."""
        s = ServeStats()
        st = load_library().hptt_cuda_server_run_poisson(
            self._h, _handles(pool), len(pool), float(rate), float(seconds), int(seed),
            float(drain_timeout), ctypes.byref(s))
        if st != 0:
            raise HpttError(st, "server_run_poisson")
        return s.as_dict()

    def destroy(self) -> None:
        if getattr(self, "_h", None):
            load_library().hptt_cuda_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


# --------------------------------------------------------------------------
# Tensor contraction through the transposes (hptt_cuda_contract_*)
# --------------------------------------------------------------------------
def _i32(v: Sequence[int]):
    return (ctypes.c_int32 * max(1, len(v)))(*[int(x) for x in v])


def _label_codes(*lists):
    """Map arbitrary hashable labels (characters, ints) to int32 codes."""
    codes = {}
    out = []
    for lst in lists:
        out.append([codes.setdefault(x, len(codes)) for x in lst])
    return out


def parse_spec(spec: str):
    """'acid,dbcj->abij' -> (labels_a, labels_b, labels_c), one character per
    dimension, fastest (stride-1) dimension first."""
    lhs, arrow, rhs = spec.replace(" ", "").partition("->")
    ops = lhs.split(",")
    if not arrow or len(ops) != 2:
        raise ValueError(f"contraction spec needs the form 'ab,bc->ac': {spec!r}")
    return list(ops[0]), list(ops[1]), list(rhs)


class Contraction:
    """C[lc] = alpha * sum_K A[la] * B[lb] + beta * C[lc] on the device:
    transposes (this library's kernels), one strided-batched cuBLAS GEMM and
    an output transpose that applies alpha and beta."""

    def __init__(self, handle: int, dtype: int, keep=()):
        self._h = ctypes.c_void_p(handle)
        self.dtype = dtype
        self._keep = keep

    def exec(self) -> None:
        self._check(load_library().hptt_cuda_contract_exec(self._h), "exec")

    def __call__(self) -> None:
        self.exec()

    def exec_on(self, stream) -> None:
        self._check(load_library().hptt_cuda_contract_exec_on(self._h, _stream_ptr(stream)),
                    "exec_on")

    def reset_data(self, A, B, C) -> None:
        self._keep = (A, B, C) + tuple(self._keep[3:])
        self._check(load_library().hptt_cuda_contract_reset_data(
            self._h, _device_ptr(A), _device_ptr(B), _device_ptr(C)), "reset_data")

    def set_coef(self, alpha, beta, complex_scalars: Optional[bool] = None) -> None:
        if complex_scalars is None:
            complex_scalars = isinstance(alpha, complex) or isinstance(beta, complex)
        self._check(load_library().hptt_cuda_contract_set_coef(
            self._h, _scalar(alpha), _scalar(beta), int(bool(complex_scalars))), "set_coef")

    def set_stream(self, stream) -> None:
        self._check(load_library().hptt_cuda_contract_set_stream(self._h, _stream_ptr(stream)),
                    "set_stream")

    def set_graph(self, on: bool) -> None:
        self._check(load_library().hptt_cuda_contract_set_graph(self._h, int(bool(on))),
                    "set_graph")

    def sync(self) -> None:
        self._check(load_library().hptt_cuda_contract_sync(self._h), "sync")

    def info(self) -> dict:
        st = ContractStats()
        self._check(load_library().hptt_cuda_contract_info(self._h, ctypes.byref(st)), "info")
        return st.as_dict()

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(4096)
        self._check(load_library().hptt_cuda_contract_describe(self._h, buf, 4096), "describe")
        return buf.value.decode()

    def destroy(self) -> None:
        if self._h.value:
            load_library().hptt_cuda_contract_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @staticmethod
    def _check(st: int, what: str) -> None:
        if st != 0:
            raise HpttError(st, "contraction " + what)


def inspect_contraction(dtype, size_a: Sequence[int], labels_a, size_b: Sequence[int],
                        labels_b, labels_c):
    """Host-only: the layout the contraction would use and its workspace
    bytes (no device, no data)."""
    la, lb, lc = _label_codes(labels_a, labels_b, labels_c)
    lib = load_library()
    buf = ctypes.create_string_buffer(4096)
    ws = ctypes.c_uint64(0)
    st = lib.hptt_cuda_contract_inspect(dtype_code(dtype), len(la), _u32(size_a), _i32(la),
                                        len(lb), _u32(size_b), _i32(lb), len(lc), _i32(lc),
                                        buf, 4096, ctypes.byref(ws))
    if st != 0:
        raise HpttError(st, "inspect_contraction")
    return buf.value.decode(), ws.value


def create_contraction(A, B, C, size_a: Sequence[int], labels_a, size_b: Sequence[int],
                       labels_b, labels_c, alpha=1.0, beta=0.0, dtype=None,
                       complex_scalars: Optional[bool] = None, workspace=None,
                       workspace_bytes: int = 0, use_graph: bool = True) -> Contraction:
    """Plan C[labels_c] = alpha * sum A[labels_a] * B[labels_b] + beta * C.

    Sizes are column-major extents (stride-1 dimension first); labels are
    any hashable values (one per dimension).  ``workspace`` (a device buffer
    of at least ``inspect_contraction(...)[1]`` bytes) avoids the plan's own
    allocation."""
    code = dtype_code(dtype if dtype is not None else A)
    la, lb, lc = _label_codes(labels_a, labels_b, labels_c)
    if complex_scalars is None:
        complex_scalars = code in (C64, C128) and (
            isinstance(alpha, complex) or isinstance(beta, complex))
    lib = load_library()
    h = ctypes.c_void_p(0)
    ws_ptr = _device_ptr(workspace) if workspace is not None else None
    if workspace is not None and not workspace_bytes:
        workspace_bytes = int(workspace.numel() * workspace.element_size())
    st = lib.hptt_cuda_contract_create(
        code, len(la), _u32(size_a), _i32(la), len(lb), _u32(size_b), _i32(lb), len(lc),
        _i32(lc), _scalar(alpha), _scalar(beta), int(bool(complex_scalars)),
        _device_ptr(A), _device_ptr(B), _device_ptr(C), ws_ptr, int(workspace_bytes),
        ctypes.byref(h))
    if st != 0:
        raise HpttError(st, "create_contraction")
    c = Contraction(h.value, code, keep=(A, B, C, workspace))
    if not use_graph:
        c.set_graph(False)
    return c


def contract(spec: str, A, B, C, size_a: Sequence[int], size_b: Sequence[int],
             alpha=1.0, beta=0.0, **kw) -> Contraction:
    """``create_contraction`` from an index string, e.g. ``'acid,dbcj->abij'``
    (one character per dimension, stride-1 dimension first)."""
    la, lb, lc = parse_spec(spec)
    return create_contraction(A, B, C, size_a, la, size_b, lb, lc, alpha, beta, **kw)


def tune_cache_load(path: Optional[str] = None) -> None:
    """Merge the autotune entries of a cache file (None: the file named by
    HPTT_B200_TUNE_CACHE)."""
    st = load_library().hptt_cuda_tune_cache_load(path.encode() if path else None)
    if st != 0:
        raise HpttError(st, f"tune_cache_load({path})")


def tune_cache_save(path: Optional[str] = None) -> None:
    """Write every autotune entry to `path` (None: HPTT_B200_TUNE_CACHE)."""
    st = load_library().hptt_cuda_tune_cache_save(path.encode() if path else None)
    if st != 0:
        raise HpttError(st, f"tune_cache_save({path})")


def tune_cache_clear() -> None:
    load_library().hptt_cuda_tune_cache_clear()


def tune_cache_size() -> int:
    n = ctypes.c_uint32(0)
    load_library().hptt_cuda_tune_cache_size(ctypes.byref(n))
    return int(n.value)


def version() -> str:
    return load_library().hptt_cuda_version().decode()
