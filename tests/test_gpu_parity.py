"""GPU parity: the sm_100a kernels, called through the C ABI, against the
oracle (itself pinned to the reference) -- bit-exact for every element type,
including the scaled cases (products and sums are rounded separately on both
sides, no FMA), NaN matching NaN.

The benchmark's workloads are checked at full size, element for element:
every sweep transpose (both scalar variants, with the shipped tuned tiles),
the plain single transpose and the hard layouts; a permute/inverse-permute
round trip adds a size-independent property.
"""
import numpy as np
import pytest

import oracle
from golden.make_golden import load as load_golden
from helpers import assert_same, footprint, gpu_run, oracle_run, random_perm, seeded

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import hptt_b200 as h  # noqa: E402

DTYPES = ["f32", "f64", "c64", "c128"]
SCALARS = [(1.0, 0.0), (2.3, 4.2), (-0.5, 1e-17), (0.0, 1.0)]


@pytest.mark.parametrize("case", list(load_golden()), ids=lambda c: c["key"])
def test_golden_fixtures(case):
    name = case["dtype"]
    got = gpu_run(name, case["in_size"], case["perm"], case["alpha"], case["beta"],
                  case["a"], case["b0"])
    assert_same(got, case["b1"], name, f"golden {case['key']}")


def _check(name, size, perm, al, be, io=None, oo=None, cs=None, seed=0, offset=0):
    rng = np.random.default_rng(seed)
    n_in, n_out = footprint(size, perm, io, oo)
    a = seeded(rng, n_in, name)
    b0 = seeded(rng, n_out, name)
    want = oracle_run(name, size, perm, al, be, a, b0, io, oo, complex_scalars=cs)
    got = gpu_run(name, size, perm, al, be, a, b0, io, oo, complex_scalars=cs,
                  device_offset_bytes=offset)
    assert_same(got, want, name, f"{name} {size} {perm} a={al} b={be} io={io} oo={oo}")


@pytest.mark.parametrize("seed", range(48))
def test_random_shapes(seed):
    rng = np.random.default_rng(1000 + seed)
    name = DTYPES[seed % 4]
    rank = 2 + seed % 5
    size = [int(x) for x in np.exp(rng.uniform(0, np.log(60), rank)).astype(int) + 1]
    while np.prod(size) > 400000:
        size[int(np.argmax(size))] //= 2
    perm = random_perm(rng, rank)
    al, be = SCALARS[seed % len(SCALARS)]
    _check(name, size, perm, al, be, seed=seed)


@pytest.mark.parametrize("name", DTYPES)
@pytest.mark.parametrize("perm", [[1, 0, 2], [2, 1, 0], [0, 2, 1], [1, 2, 0], [2, 0, 1]])
def test_all_rank3_perms_ragged(name, perm):
    _check(name, [37, 29, 23], perm, 2.3, 4.2)
    _check(name, [37, 29, 23], perm, 1.0, 0.0)


@pytest.mark.parametrize("name", DTYPES)
def test_all_rank4_perms(name):
    import itertools
    for i, perm in enumerate(itertools.permutations(range(4))):
        al, be = SCALARS[i % 2]
        _check(name, [5, 7, 3, 6], list(perm), al, be, seed=i)


@pytest.mark.parametrize("name", DTYPES)
@pytest.mark.parametrize("lead", [1, 2, 3, 4, 8, 16, 31])
def test_tiny_leading_extents(name, lead):
    _check(name, [lead, 300, 7], [1, 2, 0], 2.3, 4.2)
    _check(name, [300, lead, 7], [1, 0, 2], 1.0, 0.0)
    _check(name, [lead, 40, 9, 5], [0, 2, 3, 1], 2.3, 4.2)  # shared stride-1


@pytest.mark.parametrize("name", DTYPES)
def test_outer_sizes(name):
    _check(name, [5, 6, 7], [2, 0, 1], 2.3, 4.2, io=[8, 6, 9])
    _check(name, [5, 6, 7], [2, 0, 1], 1.0, 0.0, oo=[9, 8, 10])
    _check(name, [5, 6, 7], [0, 2, 1], 2.3, 4.2, io=[6, 7, 7], oo=[7, 7, 8])
    _check(name, [64, 6, 7], [0, 1, 2], 2.3, 4.2, io=[66, 6, 7], oo=[65, 7, 7])


@pytest.mark.parametrize("name", ["c64", "c128"])
def test_complex_scalars(name):
    _check(name, [8, 64, 4, 6, 2, 3], [5, 2, 0, 4, 1, 3], 1.5 - 0.5j, 0.25 + 1j, cs=True)
    _check(name, [8, 64, 4, 6, 2, 3], [0, 3, 2, 1, 4, 5], 1.5 - 0.5j, 0.25 + 1j, cs=True)
    _check(name, [33, 17], [1, 0], 1.5 - 0.5j, 0.0, cs=True)


@pytest.mark.parametrize("name", DTYPES)
def test_misaligned_pointers(name):
    # one element off a 16-byte boundary: vector row path must fall back
    _check(name, [64, 32, 5], [0, 2, 1], 2.3, 4.2, offset={"f32": 4, "f64": 8, "c64": 8, "c128": 16}[name])
    _check(name, [64, 32, 5], [0, 2, 1], 1.0, 0.0, offset={"f32": 4, "f64": 8, "c64": 8, "c128": 16}[name])


@pytest.mark.parametrize("name", ["f32", "f64"])
def test_special_values(name):
    rng = np.random.default_rng(5)
    size, perm = [17, 19, 3], [2, 0, 1]
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    a[::7] = np.inf
    a[1::11] = -np.inf
    a[2::13] = np.nan
    a[3::5] = -0.0
    b0 = seeded(rng, n, name)
    b0[::3] = np.nan
    for al, be in [(1.0, 0.0), (2.3, 4.2), (-1.0, 1e-20), (0.0, 0.0)]:
        want = oracle_run(name, size, perm, al, be, a, b0)
        got = gpu_run(name, size, perm, al, be, a, b0)
        assert_same(got, want, name, f"special a={al} b={be}")


@pytest.mark.parametrize("name", ["c64", "c128"])
def test_special_values_complex(name):
    """Complex elements with -0, +-Inf and NaN in either part, under complex
    scalars (1+0i with beta 0 is NOT a copy in the stated arithmetic:
    fl(fl(1*xr) - fl(0*xi)) turns -0 into +0 when xi < 0, and an infinite
    part makes the other one NaN) and under real scalars."""
    rng = np.random.default_rng(6)
    size, perm = [17, 19, 3], [2, 0, 1]
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    ar = a.view(np.float32 if name == "c64" else np.float64)
    ar[0::14] = -0.0            # real parts -0
    ar[3::22] = -0.0            # imaginary parts -0
    ar[5::26] = np.inf
    ar[8::30] = -np.inf
    ar[11::34] = np.nan
    ar[1::18] = -np.abs(ar[1::18])
    b0 = seeded(rng, n, name)
    b0.view(ar.dtype)[::5] = np.nan
    for al, be, cs in [(1 + 0j, 0j, True), (1.0, 0.0, False), (1 + 0j, 1e-20 + 0j, True),
                       (1.5 - 0.5j, 0.25 + 1j, True), (0j, 0j, True), (-1 + 0j, 0j, True),
                       (2.3, 4.2, False), (0 + 1j, 0j, True)]:
        want = oracle_run(name, size, perm, al, be, a, b0, complex_scalars=cs)
        got = gpu_run(name, size, perm, al, be, a, b0, complex_scalars=cs)
        assert_same(got, want, name, f"special a={al} b={be} complex scalars={cs}")


# Ranks 7 and 8 (the reference generates them when built with a larger
# HPTT_CODE_GEN_TRANS_ORDER_MAX, README.md:38-46); no pair of neighbouring
# output dims fuses, so the kernels see rank 7 and 8 problems.
HIGH_RANK = [
    ("f32", [3, 4, 2, 5, 3, 2, 4], [6, 4, 2, 0, 5, 3, 1]),
    ("f64", [5, 3, 7, 2, 4, 3, 6], [3, 0, 6, 2, 5, 1, 4]),
    ("c64", [2, 3, 4, 2, 3, 2, 5, 3], [7, 5, 3, 1, 6, 4, 2, 0]),
    ("c128", [5, 7, 3, 4, 6, 3, 2, 5], [1, 5, 0, 7, 3, 6, 2, 4]),
    ("f32", [33, 2, 3, 4, 2, 3, 2, 17], [0, 5, 2, 7, 4, 1, 6, 3]),
    ("f64", [9, 4, 3, 2, 5, 2, 3, 11], [7, 2, 5, 0, 3, 6, 1, 4]),
    ("f32", [40, 3, 5, 2, 7, 3, 2, 30], [7, 0, 2, 4, 6, 1, 3, 5]),
]


@pytest.mark.parametrize("name,size,perm", HIGH_RANK)
@pytest.mark.parametrize("al,be", [(1.0, 0.0), (2.3, 4.2)])
def test_ranks_7_and_8(name, size, perm, al, be):
    assert "fused rank: %d" % len(size) in h.inspect_plan(name, size, perm)
    _check(name, size, perm, al, be)


def test_identity_and_single_element():
    _check("f32", [1000, 3, 5], [0, 1, 2], 2.3, 4.2)
    _check("c128", [1, 1], [1, 0], 2.3, 4.2)
    _check("f64", [1, 1, 1, 1, 1, 1], [5, 4, 3, 2, 1, 0], 2.3, 4.2)


def test_reset_data_set_coef_and_streams():
    name = "f32"
    size, perm = [300, 200], [1, 0]
    rng = np.random.default_rng(3)
    n = 60000
    a1, a2 = seeded(rng, n, name), seeded(rng, n, name)
    b0 = seeded(rng, n, name)
    da1 = torch.from_numpy(a1).cuda()
    da2 = torch.from_numpy(a2).cuda()
    db1 = torch.from_numpy(b0.copy()).cuda()
    db2 = torch.from_numpy(b0.copy()).cuda()
    plan = h.create_plan(da1, db1, size, perm, 2.3, 4.2, 0)
    plan.exec()
    plan.reset_data(da2, db2)
    s = torch.cuda.Stream()
    plan.set_stream(s)
    plan.exec()
    plan.sync()
    assert_same(db1.cpu().numpy(), oracle_run(name, size, perm, 2.3, 4.2, a1, b0), name, "first")
    assert_same(db2.cpu().numpy(), oracle_run(name, size, perm, 2.3, 4.2, a2, b0), name, "reset")
    plan.set_coef(1.0, 0.0)
    plan.exec_on(s)
    s.synchronize()
    assert_same(db2.cpu().numpy(), oracle_run(name, size, perm, 1.0, 0.0, a2, b0), name, "coef")
    plan.set_thread_ids([0, 1])
    plan.unset_thread_ids()
    assert "fused rank" in plan.describe()


@pytest.mark.parametrize("name", ["f32", "f64"])
def test_set_coef_switches_update(name):
    """set_coef moving beta between zero and non-zero changes whether B is
    read, and with it the tile shape: the plan re-plans its tiles."""
    size, perm = [700, 90, 33], [2, 0, 1]
    rng = np.random.default_rng(21)
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    b0 = seeded(rng, n, name)
    da = torch.from_numpy(a).cuda()
    db = torch.from_numpy(b0.copy()).cuda()
    plan = h.create_plan(da, db, size, perm, 1.0, 0.0, 0)
    before = plan.describe()
    plan.set_coef(2.3, 4.2)
    after = plan.describe()
    db.copy_(torch.from_numpy(b0))
    plan.exec()
    plan.sync()
    assert_same(db.cpu().numpy(), oracle_run(name, size, perm, 2.3, 4.2, a, b0), name,
                f"update after set_coef ({before} -> {after})")
    plan.set_coef(-0.5, 0.0)
    plan.exec()
    plan.sync()
    assert_same(db.cpu().numpy(), oracle_run(name, size, perm, -0.5, 0.0, a, b0), name,
                "scale after set_coef")


def test_tuned_plan_matches():
    _check("f64", [96, 80, 12], [2, 0, 1], 2.3, 4.2)
    rng = np.random.default_rng(9)
    size, perm = [96, 80, 12], [2, 0, 1]
    n = int(np.prod(size))
    a, b0 = seeded(rng, n, "f64"), seeded(rng, n, "f64")
    got = gpu_run("f64", size, perm, 2.3, 4.2, a, b0, tuning_timeout=-1.0)
    assert_same(got, oracle_run("f64", size, perm, 2.3, 4.2, a, b0), "f64", "tuned")


# Shapes whose tiles have two-dim sides (walked or read from tables) or
# single-dim sides with an update (exact trip counts or the predicated path).
FORM_SHAPES = [
    ("f32", [30, 4, 34, 6, 5, 3], [2, 5, 1, 4, 0, 3]),
    ("f32", [54, 19, 6, 5, 4, 7], [3, 1, 5, 2, 4, 0]),
    ("f64", [17, 50, 46, 3, 2, 4], [4, 2, 3, 5, 1, 0]),
    ("f32", [65, 448, 17], [1, 0, 2]),
    ("f32", [49, 88, 93, 6], [1, 3, 0, 2]),
    ("c64", [12, 4, 4, 11, 19, 13], [4, 0, 5, 3, 1, 2]),
    ("c128", [6, 6, 15, 77, 6, 3], [1, 2, 5, 0, 3, 4]),
    ("f64", [37, 29, 23], [2, 1, 0]),
    ("c128", [33, 17, 5], [1, 0, 2]),
    ("c64", [70, 41], [1, 0]),
    ("f32", [300, 7, 13], [2, 0, 1]),
    ("f32", [1000, 333], [1, 0]),
]


@pytest.mark.parametrize("name,size,perm", FORM_SHAPES)
@pytest.mark.parametrize("al,be", [(1.0, 0.0), (2.3, 4.2)])
def test_tile_forms_match(tmp_path, name, size, perm, al, be):
    """The tuner's alternative tile forms, each forced through the tune cache
    (tune once, rewrite the entry's walk / upd_exact / threads / grid-order
    fields, reload): every form bit-exact against the oracle."""
    rng = np.random.default_rng(17)
    n_in, n_out = footprint(size, perm)
    a = seeded(rng, n_in, name)
    b0 = seeded(rng, n_out, name)
    want = oracle_run(name, size, perm, al, be, a, b0)
    h.tune_cache_clear()
    try:
        got = gpu_run(name, size, perm, al, be, a, b0, tuning_timeout=-1.0)
        assert_same(got, want, name, f"tuned {size} {perm}")
        path = tmp_path / "forms.cache"
        h.tune_cache_save(str(path))
        (line,) = path.read_text().splitlines()
        key, fields = line.split("|")
        f = fields.split()
        assert len(f) == 19
        for walk, exact, nt, order in ((0, 0, 256, 0), (0, 1, 256, 0), (1, 0, 256, 0),
                                       (1, 1, 256, 1), (1, 1, 512, 0), (0, 0, 512, 1)):
            f[7], f[8], f[9], f[10] = str(walk), str(exact), str(nt), str(order)
            f[11] = "0"  # the shared-memory tile forms, not the vector tile
            f[16] = "0"  # nor the TMA tile
            path.write_text(key + "|" + " ".join(f) + "\n")
            h.tune_cache_clear()
            h.tune_cache_load(str(path))
            got = gpu_run(name, size, perm, al, be, a, b0)
            assert_same(got, want, name,
                        f"{size} {perm} walk={walk} exact={exact} nt={nt} order={order}")
    finally:
        h.tune_cache_clear()


# --------------------------------------------------------------------------
# Workloads at full size
# --------------------------------------------------------------------------
def test_plain_single_transpose_full_size():
    """f32 {256,256,256}, perm {2,1,0}, alpha 2.3, beta 4.2, seed 0: bit-exact."""
    name, size, perm = "f32", [256, 256, 256], [2, 1, 0]
    rng = np.random.default_rng(0)
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    b0 = seeded(rng, n, name)
    got = gpu_run(name, size, perm, 2.3, 4.2, a, b0)
    want = oracle_run(name, size, perm, 2.3, 4.2, a, b0)
    assert_same(got, want, name, "plain single transpose")


@pytest.mark.parametrize("name,perm", [("c64", [5, 2, 0, 4, 1, 3]), ("c64", [0, 3, 2, 1, 4, 5]),
                                       ("c128", [5, 2, 0, 4, 1, 3]), ("c128", [0, 3, 2, 1, 4, 5])])
def test_hard_layouts_full_size(name, perm):
    size = [8, 64, 4, 64, 16, 16] if name == "c64" else [8, 64, 4, 64, 16, 8]
    rng = np.random.default_rng(3)
    n = int(np.prod(size))
    a = seeded(rng, n, name)
    b0 = seeded(rng, n, name)
    al, be = 1.5 - 0.5j, 0.25 + 1j
    got = gpu_run(name, size, perm, al, be, a, b0, complex_scalars=True)
    want = oracle_run(name, size, perm, al, be, a, b0, complex_scalars=True)
    assert_same(got, want, name, f"hard layout {perm}")


def _device_inputs(name, n, seed):
    """A and B0 made on the GPU from a seeded generator (uniform[-1, 1]), and
    page-aligned host copies of both for the oracle."""
    tdt = {"f32": torch.float32, "f64": torch.float64}[name]
    g = torch.Generator(device="cuda").manual_seed(seed)
    da = torch.rand(n, dtype=tdt, device="cuda", generator=g) * 2 - 1
    db0 = torch.rand(n, dtype=tdt, device="cuda", generator=g) * 2 - 1
    a = oracle.aligned_empty(n, oracle.NP_DTYPES[name])
    b0 = oracle.aligned_empty(n, oracle.NP_DTYPES[name])
    a[:] = da.cpu().numpy()
    b0[:] = db0.cpu().numpy()
    return da, db0, a, b0


@pytest.fixture
def shipped_tune_cache():
    """The tiles the benchmark runs: the shipped B200 autotune cache."""
    import os
    path = os.path.join(os.path.dirname(h.__file__), "tune", "b200.cache")
    h.tune_cache_clear()
    if os.path.exists(path):
        h.tune_cache_load(path)
    yield
    h.tune_cache_clear()


@pytest.mark.parametrize("idx", range(48))
def test_sweep_cases_full_size(idx, shipped_tune_cache):
    """Every transpose the benchmark times, at its full size (~200 MB per
    tensor) and with the tiles it runs: both scalar variants, every element
    compared with the oracle, bit for bit."""
    from hptt_b200.workloads import sweep_cases
    case = sweep_cases()[idx]
    name, size, perm = case["dtype"], case["in_size"], case["perm"]
    n = int(np.prod(size))
    da, db0, a, b0 = _device_inputs(name, n, 100 + idx)
    for al, be in ((1.0, 0.0), (2.3, 4.2)):
        db = db0.clone()
        plan = h.create_plan(da, db, size, perm, al, be, 0)
        assert plan is not None
        plan.exec()
        plan.sync()
        got = db.cpu().numpy()
        plan.destroy()
        del db
        want = oracle_run(name, size, perm, al, be, a, b0)
        assert_same(got, want, name, f"sweep case {idx} {size} {perm} a={al} b={be}")


def _round_trip(name, size, perm):
    """alpha=1, beta=0 is a pure permutation: perm then inverse returns A."""
    tdt = {"f32": torch.float32, "f64": torch.float64}[name]
    n = int(np.prod(size))
    g = torch.Generator(device="cuda").manual_seed(7)
    a = torch.rand(n, dtype=tdt, device="cuda", generator=g) * 2 - 1
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    out_size = [size[p] for p in perm]
    inv = [0] * len(perm)
    for k, p in enumerate(perm):
        inv[p] = k
    p1 = h.create_plan(a, b, size, perm, 1.0, 0.0, 0)
    p2 = h.create_plan(b, c, out_size, inv, 1.0, 0.0, 0)
    p1.exec()
    p2.exec()
    p2.sync()
    assert torch.equal(a.view(torch.int32 if name == "f32" else torch.int64),
                       c.view(torch.int32 if name == "f32" else torch.int64))
    # a permutation keeps the multiset of values
    assert torch.equal(torch.sort(a).values, torch.sort(b).values)
    return a, b


def test_round_trip_full_size():
    """alpha=1, beta=0 of a sweep shape and its inverse return A exactly."""
    from hptt_b200.workloads import sweep_cases
    case = sweep_cases()[44]
    _round_trip(case["dtype"], case["in_size"], case["perm"])
