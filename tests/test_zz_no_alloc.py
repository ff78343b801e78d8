"""The allocation-free entry point, hptt_cuda_transpose_noalloc.

Some callers cannot allocate device memory at the moment they transpose:
frameworks that hand out device memory only from their own pool or arena,
jobs held to a fixed device-memory budget.  For them the offset tables go
into a fixed array compiled into the library instead of a cudaMalloc'd
buffer.  Its results must equal those of the plan-based entry point
(hptt_cuda_plan_create + hptt_cuda_plan_exec) and of the oracle bit for bit,
also on consecutive calls that reuse the shared array.

The file name makes pytest collect it last, so a run that stops at its first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from helpers import assert_same, footprint, gpu_run, oracle_run, seeded

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import hptt_b200 as h  # noqa: E402


def _noalloc_fn():
    lib = h.load_library()
    f = lib.hptt_cuda_transpose_noalloc
    u32p = ctypes.POINTER(ctypes.c_uint32)
    dp = ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_int, ctypes.c_uint32, u32p, u32p, u32p, u32p, dp, dp, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _u32(v):
    return (ctypes.c_uint32 * len(v))(*v) if v is not None else None


def _run_noalloc(name, size, perm, al, be, a, b0, io=None, oo=None, cs=False):
    """One call through the C ABI on the current stream; returns B on the host."""
    da = torch.from_numpy(np.asarray(a)).cuda()
    db = torch.from_numpy(np.asarray(b0).copy()).cuda()
    za, zb = complex(al), complex(be)
    alpha = (ctypes.c_double * 2)(za.real, za.imag)
    beta = (ctypes.c_double * 2)(zb.real, zb.imag)
    stream = torch.cuda.current_stream()
    rc = _noalloc_fn()(h.dtype_code(name), len(size), _u32(size), _u32(perm), _u32(io),
                       _u32(oo), alpha, beta, int(cs), da.data_ptr(), db.data_ptr(),
                       stream.cuda_stream)
    assert rc == 0, f"hptt_cuda_transpose_noalloc returned {rc}"
    stream.synchronize()
    return db.cpu().numpy()


CASES = [
    # (dtype, in_size, perm, alpha, beta, in_outer, out_outer, complex scalars)
    ("f32", [256, 96, 40], [2, 1, 0], 2.3, 4.2, None, None, False),       # tile kernel
    ("c128", [8, 6, 4, 6, 4, 3], [5, 2, 0, 4, 1, 3], 1.5 - 0.5j, 0.25 + 1j, None, None, True),
    ("f64", [300, 17, 9], [0, 2, 1], 1.0, 0.0, None, None, False),       # row kernel
    ("f32", [37, 29, 23], [1, 2, 0], -0.5, 1.0, [40, 29, 25], None, False),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{len(c[1])}d")
def test_noalloc_matches_plan_twice(case):
    name, size, perm, al, be, io, oo, cs = case
    rng = np.random.default_rng(11)
    n_in, n_out = footprint(size, perm, io, oo)
    for call in range(2):  # the second call reuses the shared table array
        a = seeded(rng, n_in, name)
        b0 = seeded(rng, n_out, name)
        want = gpu_run(name, size, perm, al, be, a, b0, io, oo, complex_scalars=cs)
        got = _run_noalloc(name, size, perm, al, be, a, b0, io, oo, cs)
        assert_same(got, want, name, f"no-alloc call {call}")
        ref = oracle_run(name, size, perm, al, be, a, b0, io, oo, complex_scalars=cs)
        assert_same(got, ref, name, f"no-alloc call {call} vs oracle")


def test_noalloc_alternating_shapes():
    """Two different problems back to back: the second call must not see the
    first call's tables."""
    rng = np.random.default_rng(12)
    for name, size, perm in (("f32", [64, 48, 20], [1, 2, 0]), ("f64", [9, 70, 33], [2, 0, 1])):
        a = seeded(rng, int(np.prod(size)), name)
        b0 = seeded(rng, int(np.prod(size)), name)
        want = gpu_run(name, size, perm, 2.3, 4.2, a, b0)
        got = _run_noalloc(name, size, perm, 2.3, 4.2, a, b0)
        assert_same(got, want, name, f"alternating {size}")
        assert_same(got, oracle_run(name, size, perm, 2.3, 4.2, a, b0), name,
                    f"alternating {size} vs oracle")


def test_noalloc_rejects_bad_arguments():
    f = _noalloc_fn()
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    assert f(0, 2, _u32([4, 4]), _u32([1, 1]), None, None, one, zero, 0, 0x1000, 0x2000,
             None) == 5
    assert f(0, 2, _u32([4, 4]), _u32([1, 0]), None, None, one, zero, 0, None, 0x2000,
             None) == 1
    size_fn = h.load_library().hptt_cuda_noalloc_table_bytes
    size_fn.restype = ctypes.c_size_t
    assert size_fn() == 65536


def test_noalloc_tma_tile_from_cache(tmp_path):
    """A tune-cache entry that names the TMA tile: the allocation-free call
    runs it (persistent and one-CTA-per-tile forms) on 16-byte aligned bases
    and plans the element tile on bases one element off, equal to the oracle
    either way."""
    name, size, perm, al, be = "f32", [100, 36, 60], [1, 0, 2], 2.3, 4.2
    esz = 4
    rng = np.random.default_rng(29)
    n_in, n_out = footprint(size, perm)
    a = seeded(rng, n_in, name)
    b0 = seeded(rng, n_out, name)
    want = oracle_run(name, size, perm, al, be, a, b0)
    h.tune_cache_clear()
    try:
        x = torch.zeros(n_in, dtype=torch.float32, device="cuda")
        y = torch.zeros(n_out, dtype=torch.float32, device="cuda")
        p = h.create_plan(x, y, size, perm, al, be, 1, 2e-3, dtype=name)
        assert p is not None
        p.destroy()
        path = tmp_path / "noalloc_tt.cache"
        h.tune_cache_save(str(path))
        (line,) = path.read_text().splitlines()
        key, fields = line.split("|")
        f = fields.split()
        assert len(f) == 19
        for stages, kx, ky in ((1, 2, 1), (3, 1, 1)):
            f[10], f[11] = "0", "0"
            f[16:19] = [str(stages), str(kx), str(ky)]
            path.write_text(key + "|" + " ".join(f) + "\n")
            h.tune_cache_clear()
            h.tune_cache_load(str(path))
            for offset in (0, 1):
                da = torch.empty(n_in + offset, dtype=torch.float32, device="cuda")
                db = torch.empty(n_out + offset, dtype=torch.float32, device="cuda")
                da[offset:].copy_(torch.from_numpy(a))
                db[offset:].copy_(torch.from_numpy(b0))
                alpha = (ctypes.c_double * 2)(al, 0.0)
                beta = (ctypes.c_double * 2)(be, 0.0)
                stream = torch.cuda.current_stream()
                rc = _noalloc_fn()(h.dtype_code(name), len(size), _u32(size), _u32(perm), None,
                                   None, alpha, beta, 0, da[offset:].data_ptr(),
                                   db[offset:].data_ptr(), stream.cuda_stream)
                assert rc == 0
                stream.synchronize()
                assert_same(db[offset:].cpu().numpy(), want, name,
                            f"stages={stages} boxes={kx}x{ky} offset={offset * esz} B")
    finally:
        h.tune_cache_clear()
