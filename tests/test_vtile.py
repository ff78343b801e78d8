"""GPU parity of the vector tile (16-byte windows on both sides of the
shared-memory transpose), forced through the tune cache on shapes with odd
extents, multi-dim runs and edge tiles, with base pointers on and off a
16-byte boundary, against the oracle bit for bit."""
import numpy as np
import pytest

from helpers import assert_same, footprint, oracle_run, seeded

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import hptt_b200 as h  # noqa: E402

TDT = {"f32": torch.float32, "f64": torch.float64, "c64": torch.complex64}
ESZ = {"f32": 4, "f64": 8, "c64": 8}

SHAPES = [
    ("f32", [500, 333], [1, 0]),                    # odd extents, both sides chunked
    ("f32", [37, 29, 23], [2, 1, 0]),               # every tile an edge tile
    ("f64", [233, 66, 17], [1, 0, 2]),
    ("c64", [70, 41], [1, 0]),
    ("f32", [30, 4, 34, 6, 5, 3], [2, 5, 1, 4, 0, 3]),  # two-dim X and Y runs (tables)
    ("f32", [4, 6, 101, 57, 4], [4, 2, 3, 0, 1]),   # tiny output run
    ("f64", [17, 20, 46, 3, 2, 4], [4, 2, 3, 5, 1, 0]),
    ("c64", [5, 3, 7, 40, 9], [3, 4, 0, 2, 1]),
]

# (threads, window slots per row, per column, grid order, vectors per thread,
# B read before the A loads -- update tiles of the four-vector build only)
FORMS = [(256, 16, 16, 0, 8, 0), (256, 32, 8, 1, 8, 0), (512, 32, 32, 0, 8, 0),
         (256, 8, 32, 0, 4, 0), (512, 8, 8, 1, 4, 0), (512, 16, 32, 0, 4, 0),
         (256, 16, 32, 0, 4, 1), (512, 32, 16, 1, 4, 1)]


def _run(name, size, perm, al, be, a, b0, offset, cs=None):
    off = offset // ESZ[name]
    da = torch.empty(a.size + off, dtype=TDT[name], device="cuda")
    db = torch.empty(b0.size + off, dtype=TDT[name], device="cuda")
    da[off:].copy_(torch.from_numpy(np.asarray(a)))
    db[off:].copy_(torch.from_numpy(np.asarray(b0)))
    plan = h.create_plan(da[off:], db[off:], size, perm, al, be, 1, dtype=name,
                         complex_scalars=cs)
    assert plan is not None
    desc = plan.describe()
    plan.exec()
    plan.sync()
    out = db[off:].cpu().numpy()
    plan.destroy()
    return out, desc


def _cache_line(tmp_path, name, size, perm, al, be, cs):
    """The tune-cache line of this problem (one quick tuning pass makes it)."""
    h.tune_cache_clear()
    n_in, n_out = footprint(size, perm)
    x = torch.zeros(n_in, dtype=TDT[name], device="cuda")
    y = torch.zeros(n_out, dtype=TDT[name], device="cuda")
    p = h.create_plan(x, y, size, perm, al, be, 1, 2e-3, dtype=name, complex_scalars=cs)
    assert p is not None
    p.destroy()
    path = tmp_path / "vt.cache"
    h.tune_cache_save(str(path))
    (line,) = path.read_text().splitlines()
    key, fields = line.split("|")
    f = fields.split()
    assert len(f) == 19
    return path, key, f


def _force(path, key, f, nt, nvx, nvy, order, vj=8, pre=0):
    g = list(f)
    g[9:17] = [str(nt), str(order), "1", str(nvx), str(nvy), str(vj), str(pre), "0"]
    path.write_text(key + "|" + " ".join(g) + "\n")
    h.tune_cache_clear()
    h.tune_cache_load(str(path))


SCAL = [(1.0, 0.0, None), (2.3, 4.2, None), (-0.5, 1e-17, None), (0.0, 1.0, None),
        (complex(1.5, -0.5), complex(0.25, 1.0), True), (complex(1.0, 0.0), 0.0, True)]


@pytest.mark.parametrize("name,size,perm", SHAPES)
@pytest.mark.parametrize("si", range(len(SCAL)))
def test_vector_tile_forms(tmp_path, name, size, perm, si):
    al, be, cs = SCAL[si]
    if cs and name != "c64":
        pytest.skip("complex scalars: complex elements only")
    rng = np.random.default_rng(31 + si)
    n_in, n_out = footprint(size, perm)
    a = seeded(rng, n_in, name)
    b0 = seeded(rng, n_out, name)
    want = oracle_run(name, size, perm, al, be, a, b0, complex_scalars=cs)
    try:
        path, key, f = _cache_line(tmp_path, name, size, perm, al, be, cs)
        for nt, nvx, nvy, order, vj, pre in FORMS:
            _force(path, key, f, nt, nvx, nvy, order, vj, pre)
            for offset in (0, ESZ[name], 3 * ESZ[name]):
                got, desc = _run(name, size, perm, al, be, a, b0, offset, cs)
                assert "vector tile" in desc, desc
                assert_same(got, want, name,
                            f"{size} {perm} a={al} b={be} form={nt},{nvx},{nvy},{order},{vj},{pre} "
                            f"offset={offset}")
    finally:
        h.tune_cache_clear()


def test_vector_tile_special_values(tmp_path):
    """Inf, NaN and -0 through the vector tile's scale and update paths."""
    name, size, perm = "f32", [67, 45, 9], [2, 0, 1]
    rng = np.random.default_rng(77)
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
            path, key, f = _cache_line(tmp_path, name, size, perm, al, be, None)
            _force(path, key, f, 256, 16, 16, 0)
            got, desc = _run(name, size, perm, al, be, a, b0, 4)
            assert "vector tile" in desc
            assert_same(got, want, name, f"special a={al} b={be}")
    finally:
        h.tune_cache_clear()
