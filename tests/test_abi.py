"""CPU-only checks of the C ABI library: it loads, exports every symbol the
public headers declare, and applies the reference's argument guard without a
device (create returns the reference's nullptr cases as statuses)."""
import ctypes
import os
import re

import pytest

import hptt_b200 as h

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(hptt_cuda_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_loads():
    lib = h.load_library()
    assert h.version().startswith("hptt-b200")
    assert lib is not None


@pytest.mark.parametrize("sym", declared_functions())
def test_symbol_exported(sym):
    lib = ctypes.CDLL(h.library_path())
    assert hasattr(lib, sym), f"{sym} declared in include/ but not exported"


def test_status_strings():
    lib = h.load_library()
    for st in range(0, 15):
        assert lib.hptt_cuda_status_string(st)


class _Ptr:
    """Stand-in device address for argument-guard tests (never dereferenced)."""

    def __init__(self, v):
        self.v = v

    def data_ptr(self):
        return self.v


A, B = _Ptr(0x10000), _Ptr(0x20000)

# The reference returns nullptr for each of these (inc/hptt/hptt.h:71-83).
NULL_CASES = [
    ("null in", dict(in_data=_Ptr(0))),
    ("null out", dict(out_data=_Ptr(0))),
    ("rank 1", dict(in_size=[4], perm=[0])),
    ("size length", dict(in_size=[4, 4, 4])),
    ("zero extent", dict(in_size=[4, 0])),
    ("in outer too small", dict(in_outer_size=[3, 4])),
    ("in outer length", dict(in_outer_size=[4, 4, 4])),
    ("out outer too small", dict(out_outer_size=[4, 3])),
    ("perm repeat", dict(perm=[1, 1])),
    ("perm range", dict(perm=[0, 2])),
]


@pytest.mark.parametrize("what,kw", NULL_CASES, ids=[c[0] for c in NULL_CASES])
def test_create_plan_returns_none_like_reference(what, kw):
    args = dict(in_data=A, out_data=B, in_size=[4, 5], perm=[1, 0], alpha=1.0, beta=0.0,
                num_threads=1)
    args.update(kw)
    plan = h.create_plan(args.pop("in_data"), args.pop("out_data"), args.pop("in_size"),
                         args.pop("perm"), args.pop("alpha"), args.pop("beta"),
                         args.pop("num_threads"), dtype="f32", **args)
    assert plan is None


def test_c_abi_status_codes():
    lib = h.load_library()
    u = lambda v: (ctypes.c_uint32 * len(v))(*v)  # noqa: E731
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    out = ctypes.c_void_p()
    call = lambda dtype, rank, size, perm, a, b: lib.hptt_cuda_plan_create(  # noqa: E731
        dtype, rank, u(size), u(perm), None, None, one, zero, 0, a, b, 1, 0.0,
        ctypes.byref(out))
    assert call(0, 2, [4, 4], [1, 0], None, 0x1000) == 1
    assert call(0, 1, [4], [0], 0x1000, 0x2000) == 2
    assert call(0, 2, [4, 0], [1, 0], 0x1000, 0x2000) == 4
    assert call(0, 2, [4, 4], [1, 1], 0x1000, 0x2000) == 5
    assert call(9, 2, [4, 4], [1, 0], 0x1000, 0x2000) == 6
    assert out.value is None


def test_reset_data_and_exec_reject_bad_handles():
    lib = h.load_library()
    assert lib.hptt_cuda_plan_exec(None) == 11
    assert lib.hptt_cuda_plan_destroy(None) == 11
    assert lib.hptt_cuda_plan_reset_data(None, None, None) == 11


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_valid_plan_without_device_raises():
    with pytest.raises(h.HpttError) as e:
        h.create_plan(A, B, [4, 5], [1, 0], 1.0, 0.0, 1, dtype="f32")
    assert e.value.status == 8


def test_tune_cache_round_trip(tmp_path):
    """Cache files: load merges entries (missing trailing fields -- the
    iteration cap, the whole-extent option, the grid order, the vector-tile
    switch -- read as 0, the side walk and the exact update form as 1, the
    threads per CTA as 256, the vector tile's window slots as 16 and its
    vectors per thread as 8), save
    writes every entry back, clear empties."""
    src = tmp_path / "in.cache"
    src.write_text(
        "NVIDIA B200 0 2 1,0 27 0|256 16384 32768 512 0\n"
        "NVIDIA B200 1 3 2,0,1 28 1|128 8192 32768 512 1 4\n"
        "NVIDIA B200 0 4 2,3,0,1 27 1|256 16384 32768 512 0 0 1 0\n"
        "NVIDIA B200 0 3 2,1,0 27 1|256 16384 32768 512 0 0 0 1 1 256 0 1 32 8 4\n"
        "not a cache line\n")
    h.tune_cache_clear()
    assert h.tune_cache_size() == 0
    h.tune_cache_load(str(src))
    assert h.tune_cache_size() == 4
    out = tmp_path / "out.cache"
    h.tune_cache_save(str(out))
    lines = sorted(out.read_text().splitlines())
    assert lines == ["NVIDIA B200 0 2 1,0 27 0|256 16384 32768 512 0 0 0 1 1 256 0 0 16 16 8 0 0 2 2",
                     "NVIDIA B200 0 3 2,1,0 27 1|256 16384 32768 512 0 0 0 1 1 256 0 1 32 8 4 0 0 2 2",
                     "NVIDIA B200 0 4 2,3,0,1 27 1|256 16384 32768 512 0 0 1 0 1 256 0 0 16 16 8 0 0 2 2",
                     "NVIDIA B200 1 3 2,0,1 28 1|128 8192 32768 512 1 4 0 1 1 256 0 0 16 16 8 0 0 2 2"]
    h.tune_cache_clear()
    assert h.tune_cache_size() == 0
    with pytest.raises(h.HpttError):
        h.tune_cache_load(str(tmp_path / "missing.cache"))
