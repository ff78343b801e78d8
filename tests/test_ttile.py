"""GPU parity of the TMA tile (tensor-map box loads and stores around the
shared-memory transpose), forced through the tune cache on shapes whose
strides TMA can describe -- odd extents past the 128-byte boxes, ranks 2-5,
sub-tensors -- against the oracle bit for bit, with a misaligned base
pointer falling back to the element tile, and no bounded wait running out."""
import numpy as np
import pytest

from helpers import assert_same, footprint, oracle_run, seeded

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ctypes  # noqa: E402

import hptt_b200 as h  # noqa: E402

TDT = {"f32": torch.float32, "f64": torch.float64, "c64": torch.complex64}
ESZ = {"f32": 4, "f64": 8, "c64": 8}

# (dtype, in_size, perm, in_outer, out_outer)
SHAPES = [
    ("f32", [64, 48, 20], [2, 1, 0], None, None),
    ("f32", [100, 36, 60], [1, 0, 2], None, None),
    ("f64", [30, 18, 8], [2, 0, 1], None, None),
    ("c64", [16, 5, 6, 10], [3, 1, 0, 2], None, None),
    ("f32", [1000, 332], [1, 0], None, None),
    ("f64", [258, 130], [1, 0], None, None),
    ("f32", [8, 3, 4, 5, 4], [4, 2, 0, 3, 1], None, None),  # fused rank 5
    ("f32", [40, 20, 12], [2, 0, 1], [44, 24, 12], [20, 40, 40]),
    ("c64", [6, 10, 7], [1, 2, 0], [8, 10, 9], [12, 7, 10]),
]

# (boxes along input dim 0, boxes along the output's leading dim, grid order,
# stages: 1 = one CTA per tile, 2-4 = persistent CTAs with that many tiles of
# loads in flight)
FORMS = [(1, 1, 0, 1), (2, 2, 1, 1), (4, 2, 0, 1), (1, 4, 1, 1), (2, 1, 0, 1),
         (1, 1, 0, 2), (2, 2, 1, 4), (1, 2, 0, 3), (4, 1, 1, 2), (1, 1, 1, 4)]

SCAL = [(1.0, 0.0, None), (2.3, 4.2, None), (-0.5, 1e-17, None), (0.0, 1.0, None),
        (complex(1.5, -0.5), complex(0.25, 1.0), True)]


def _timeouts():
    lib = h.load_library()
    f = lib.hptt_cuda_debug_tma_timeouts
    f.argtypes = [ctypes.POINTER(ctypes.c_uint32)]
    f.restype = ctypes.c_int
    v = ctypes.c_uint32(0)
    assert f(ctypes.byref(v)) == 0
    return v.value


def _run(name, size, perm, io, oo, al, be, a, b0, offset, cs=None):
    off = offset // ESZ[name]
    da = torch.empty(a.size + off, dtype=TDT[name], device="cuda")
    db = torch.empty(b0.size + off, dtype=TDT[name], device="cuda")
    da[off:].copy_(torch.from_numpy(np.asarray(a)))
    db[off:].copy_(torch.from_numpy(np.asarray(b0)))
    plan = h.create_plan(da[off:], db[off:], size, perm, al, be, 1, 0.0, io or (), oo or (),
                         dtype=name, complex_scalars=cs)
    assert plan is not None
    desc = plan.describe()
    plan.exec()
    plan.sync()
    out = db[off:].cpu().numpy()
    plan.destroy()
    return out, desc


def _cache_line(tmp_path, name, size, perm, io, oo, al, be, cs):
    """The tune-cache line of this problem (one quick tuning pass makes it)."""
    h.tune_cache_clear()
    n_in, n_out = footprint(size, perm, io, oo)
    x = torch.zeros(n_in, dtype=TDT[name], device="cuda")
    y = torch.zeros(n_out, dtype=TDT[name], device="cuda")
    p = h.create_plan(x, y, size, perm, al, be, 1, 2e-3, io or (), oo or (), dtype=name,
                      complex_scalars=cs)
    assert p is not None
    p.destroy()
    path = tmp_path / "tt.cache"
    h.tune_cache_save(str(path))
    (line,) = path.read_text().splitlines()
    key, fields = line.split("|")
    f = fields.split()
    assert len(f) == 19
    return path, key, f


def _force(path, key, f, kx, ky, order, stages=1):
    g = list(f)
    g[10] = str(order)
    g[11] = "0"
    g[16:19] = [str(stages), str(kx), str(ky)]
    path.write_text(key + "|" + " ".join(g) + "\n")
    h.tune_cache_clear()
    h.tune_cache_load(str(path))


@pytest.mark.parametrize("name,size,perm,io,oo", SHAPES)
@pytest.mark.parametrize("si", range(len(SCAL)))
def test_tma_tile_forms(tmp_path, name, size, perm, io, oo, si):
    al, be, cs = SCAL[si]
    if cs and name != "c64":
        pytest.skip("complex scalars: complex elements only")
    rng = np.random.default_rng(53 + si)
    n_in, n_out = footprint(size, perm, io, oo)
    a = seeded(rng, n_in, name)
    b0 = seeded(rng, n_out, name)
    want = oracle_run(name, size, perm, al, be, a, b0, in_outer=io, out_outer=oo,
                      complex_scalars=cs)
    before = _timeouts()
    try:
        path, key, f = _cache_line(tmp_path, name, size, perm, io, oo, al, be, cs)
        for kx, ky, order, stages in FORMS:
            _force(path, key, f, kx, ky, order, stages)
            # 16-byte aligned bases: the TMA tile; one element off: the
            # plan's element tile (same cache line)
            for offset in (0, ESZ[name]):
                got, desc = _run(name, size, perm, io, oo, al, be, a, b0, offset, cs)
                assert "TMA tile" in desc, desc
                assert_same(got, want, name,
                            f"{size} {perm} a={al} b={be} boxes={kx}x{ky} order={order} "
                            f"stages={stages} offset={offset}")
    finally:
        h.tune_cache_clear()
    assert _timeouts() == before


def test_tma_tile_special_values(tmp_path):
    """Inf, NaN and -0 through the TMA tile's scale and update paths."""
    name, size, perm = "f32", [132, 72, 12], [2, 0, 1]
    rng = np.random.default_rng(78)
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    a[::7] = np.inf
    a[1::11] = -np.inf
    a[2::13] = np.nan
    a[3::5] = -0.0
    b0 = seeded(rng, n, name)
    b0[::3] = np.nan
    try:
        for al, be in [(1.0, 0.0), (2.3, 4.2), (-1.0, 1e-20), (0.0, 0.0)]:
            want = oracle_run(name, size, perm, al, be, a, b0)
            path, key, f = _cache_line(tmp_path, name, size, perm, None, None, al, be, None)
            for stages in (1, 3):
                _force(path, key, f, 2, 2, 0, stages)
                got, desc = _run(name, size, perm, None, None, al, be, a, b0, 0)
                assert "TMA tile" in desc
                assert_same(got, want, name, f"special a={al} b={be} stages={stages}")
    finally:
        h.tune_cache_clear()


def test_tma_tile_plain_workload(tmp_path):
    """The plain workload's shape (f32 256^3, perm 2,1,0, update) through
    every box count and stage count the tuner tries, against the oracle
    (forms whose stages do not fit in shared memory plan another kernel)."""
    name, size, perm, al, be = "f32", [256, 256, 256], [2, 1, 0], 2.3, 4.2
    rng = np.random.default_rng(5)
    n = 256 ** 3
    a = seeded(rng, n, name)
    b0 = seeded(rng, n, name)
    want = oracle_run(name, size, perm, al, be, a, b0)
    try:
        path, key, f = _cache_line(tmp_path, name, size, perm, None, None, al, be, None)
        for kx, ky in ((1, 1), (2, 1), (1, 2), (2, 2), (4, 1), (1, 4), (4, 2), (2, 4)):
            for stages in (1, 2, 4):
                _force(path, key, f, kx, ky, 0, stages)
                got, desc = _run(name, size, perm, None, None, al, be, a, b0, 0)
                kb = kx * ky * 4096  # bytes of a tile's boxes
                fits = stages == 1 or (kx * ky <= 4 and
                                       stages * kb * 2 + 3 * kb + 1280 <= 227 * 1024)
                assert ("TMA tile" in desc) == fits, desc
                assert ("persistent" in desc) == (fits and stages > 1), desc
                assert_same(got, want, name, f"boxes={kx}x{ky} stages={stages}")
    finally:
        h.tune_cache_clear()


def _random_case(seed):
    """A seeded problem a TMA tile can serve (the CPU replay's generator):
    input dim 0 and the output's leading dim in multiples of 16 bytes."""
    rng = np.random.default_rng(seed)
    name = ["f32", "f64", "c64"][seed % 3]
    q = 4 if name == "f32" else 2
    rank = int(rng.integers(2, 6))
    while True:
        perm = [int(x) for x in rng.permutation(rank)]
        if perm[0] != 0:
            break
    size = [int(rng.integers(2, 9)) for _ in range(rank)]
    size[0] = q * int(rng.integers(1, 12))
    size[perm[0]] = q * int(rng.integers(1, 12))
    return name, size, perm


@pytest.mark.parametrize("seed", range(12))
def test_tma_tile_random_shapes(tmp_path, seed):
    name, size, perm = _random_case(seed)
    rng = np.random.default_rng(900 + seed)
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    b0 = seeded(rng, n, name)
    try:
        for al, be in ((1.0, 0.0), (2.3, 4.2)):
            want = oracle_run(name, size, perm, al, be, a, b0)
            path, key, f = _cache_line(tmp_path, name, size, perm, None, None, al, be, None)
            for kx, ky, order, stages in ((1, 1, 0, 1), (2, 1, 1, 3)):
                _force(path, key, f, kx, ky, order, stages)
                got, desc = _run(name, size, perm, None, None, al, be, a, b0, 0)
                assert "TMA tile" in desc, desc
                assert_same(got, want, name, f"seed {seed} {size} {perm} a={al} b={be} "
                                             f"boxes={kx}x{ky} stages={stages}")
    finally:
        h.tune_cache_clear()
