"""CPU replay of every launch's addressing (no GPU).

hptt_cuda_debug_check_indexing plans a problem and walks every tile and
thread with the kernels' own index helpers: all A/B/shared-memory accesses
must stay in bounds, every inner B element must be written exactly once with
the A element the permutation maps to it, and padding must stay untouched.
"""
import ctypes

import numpy as np
import pytest

import hptt_b200 as h

_u32p = ctypes.POINTER(ctypes.c_uint32)


def check(dtype, size, perm, io=None, oo=None, max_vec_bytes=0):
    lib = h.load_library()
    f = lib.hptt_cuda_debug_check_indexing
    f.argtypes = [ctypes.c_int, ctypes.c_uint32, _u32p, _u32p, _u32p, _u32p, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_uint64)]
    f.restype = ctypes.c_int
    u = lambda v: (ctypes.c_uint32 * len(v))(*v) if v is not None else None  # noqa: E731
    n = ctypes.c_uint64(0)
    rc = f(h.dtype_code(dtype), len(size), u(size), u(perm), u(io), u(oo), max_vec_bytes,
           ctypes.byref(n))
    return rc, n.value


def _random_case(seed):
    rng = np.random.default_rng(seed)
    rank = int(rng.integers(2, 7))
    dt = ["f32", "f64", "c64", "c128"][int(rng.integers(0, 4))]
    size = [int(x) for x in np.exp(rng.uniform(0, np.log(40), rank)).astype(int) + 1]
    while np.prod(size) > 80000:
        size[int(np.argmax(size))] //= 2
    perm = [int(x) for x in rng.permutation(rank)]
    io = oo = None
    if seed % 3 == 0:
        io = [s + int(rng.integers(0, 3)) for s in size]
    if seed % 5 == 0:
        # satisfy both the reference guard and the output extents
        oo = [max(size[p], size[perm[p]]) + int(rng.integers(0, 3)) for p in perm]
        oo = [max(oo[k], size[perm[k]]) for k in range(rank)]
    return dt, size, perm, io, oo


@pytest.mark.parametrize("seed", range(600))
def test_replay_random(seed):
    dt, size, perm, io, oo = _random_case(seed)
    for mv in (0, {"f32": 4, "f64": 8, "c64": 8, "c128": 16}[dt]):
        rc, n = check(dt, size, perm, io, oo, mv)
        if rc == 4:  # rejected by the reference's own outer-size guard
            pytest.skip("guard")
        assert rc == 0, (dt, size, perm, io, oo, mv, rc)
        assert n == np.prod(size)


SHAPES = [
    ("f32", [256, 256, 256], [2, 1, 0]),          # plain single transpose workload
    ("f32", [4, 100000], [1, 0]),                  # tiny input-leading extent
    ("f32", [100000, 3], [1, 0]),                  # tiny output-leading extent
    ("c64", [8, 64, 4, 64, 16, 2], [5, 2, 0, 4, 1, 3]),
    ("c128", [8, 64, 4, 64, 16, 2], [0, 3, 2, 1, 4, 5]),
    ("c64", [2, 64, 4, 16, 16, 8], [0, 3, 2, 1, 4, 5]),
    ("f64", [4097, 513], [1, 0]),
    ("f32", [7, 5, 3, 2, 11, 13], [5, 4, 3, 2, 1, 0]),
    ("f64", [3, 3, 3, 3, 3, 3], [1, 0, 3, 2, 5, 4]),
    ("f32", [1, 906, 1, 906], [2, 3, 0, 1]),
    ("f32", [1, 1], [1, 0]),
    ("c128", [1000, 7], [0, 1]),
]


@pytest.mark.parametrize("dt,size,perm", SHAPES)
def test_replay_shapes(dt, size, perm):
    # the vector limit only changes row-kernel plans (shared stride-1 dim)
    for mv in ((0, 4) if perm[0] == 0 else (0,)):
        rc, n = check(dt, size, perm, max_vec_bytes=mv)
        assert rc == 0, (dt, size, perm, mv, rc)
        assert n == np.prod(size)


# Ranks 7 and 8 (the reference generates them when built with a larger
# HPTT_CODE_GEN_TRANS_ORDER_MAX, README.md:38-46).  No two neighbouring output
# dims are consecutive input dims in order, so nothing fuses below rank 7.
HIGH_RANK = [
    ("f32", [3, 4, 2, 5, 3, 2, 4], [6, 4, 2, 0, 5, 3, 1]),
    ("f64", [5, 3, 7, 2, 4, 3, 6], [3, 0, 6, 2, 5, 1, 4]),
    ("c64", [2, 3, 4, 2, 3, 2, 5, 3], [7, 5, 3, 1, 6, 4, 2, 0]),
    ("c128", [5, 7, 3, 4, 6, 3, 2, 5], [1, 5, 0, 7, 3, 6, 2, 4]),
    ("f32", [33, 2, 3, 4, 2, 3, 2, 17], [0, 5, 2, 7, 4, 1, 6, 3]),
    ("f64", [9, 4, 3, 2, 5, 2, 3, 11], [7, 2, 5, 0, 3, 6, 1, 4]),
]


def fused_rank(dt, size, perm):
    d = h.inspect_plan(dt, size, perm)
    return int(d.split("fused rank:")[1].split()[0])


@pytest.mark.parametrize("dt,size,perm", HIGH_RANK)
def test_replay_ranks_7_and_8(dt, size, perm):
    assert fused_rank(dt, size, perm) == len(size)
    for mv in (0, {"f32": 4, "f64": 8, "c64": 8, "c128": 16}[dt]):
        rc, n = check(dt, size, perm, max_vec_bytes=mv)
        assert rc == 0, (dt, size, perm, mv, rc)
        assert n == np.prod(size)


@pytest.mark.parametrize("seed", range(60))
def test_replay_random_ranks_7_and_8(seed):
    rng = np.random.default_rng(5000 + seed)
    rank = 7 + seed % 2
    dt = ["f32", "f64", "c64", "c128"][seed % 4]
    size = [int(x) for x in np.exp(rng.uniform(np.log(2), np.log(12), rank)).astype(int)]
    while np.prod(size) > 300000:
        size[int(np.argmax(size))] //= 2
    size = [max(2, s) for s in size]
    perm = [int(x) for x in rng.permutation(rank)]
    rc, n = check(dt, size, perm)
    assert rc == 0, (dt, size, perm, rc)
    assert n == np.prod(size)


def check_vtile(dtype, size, perm, nt, nvx, nvy, order, update, mis_a, mis_b, vj=8):
    lib = h.load_library()
    f = lib.hptt_cuda_debug_check_vtile
    f.argtypes = [ctypes.c_int, ctypes.c_uint32, _u32p, _u32p, _u32p, _u32p] + \
        [ctypes.c_int] * 8 + [ctypes.POINTER(ctypes.c_uint64)]
    f.restype = ctypes.c_int
    u = lambda v: (ctypes.c_uint32 * len(v))(*v)  # noqa: E731
    n = ctypes.c_uint64(0)
    rc = f(h.dtype_code(dtype), len(size), u(size), u(perm), None, None, nt, nvx, nvy, vj,
           order, update, mis_a, mis_b, ctypes.byref(n))
    return rc, n.value


# The vector-tile shapes of the GPU tests, and small shapes with the sweep
# workload's structure (odd extents, multi-dim runs, tiny runs).
VTILE_SHAPES = [
    ("f32", [500, 333], [1, 0]),
    ("f32", [37, 29, 23], [2, 1, 0]),
    ("f64", [233, 66, 17], [1, 0, 2]),
    ("c64", [70, 41], [1, 0]),
    ("f32", [30, 4, 34, 6, 5, 3], [2, 5, 1, 4, 0, 3]),
    ("f32", [4, 6, 101, 57, 4], [4, 2, 3, 0, 1]),
    ("f64", [17, 20, 46, 3, 2, 4], [4, 2, 3, 5, 1, 0]),
    ("c64", [5, 3, 7, 40, 9], [3, 4, 0, 2, 1]),
    ("f32", [67, 45, 9], [2, 0, 1]),
    ("f32", [983, 16, 5, 3], [3, 0, 1, 2]),
    ("f32", [12, 4, 4, 11, 19, 13], [4, 0, 5, 3, 1, 2]),
    ("f64", [4, 18, 94, 7, 5], [4, 2, 0, 3, 1]),
]


@pytest.mark.parametrize("dt,size,perm", VTILE_SHAPES)
def test_replay_vtile_every_tuner_form(dt, size, perm):
    """Every window-slot shape, thread count, vectors per thread and grid
    order the autotuner times, with both update settings and base addresses
    on and off a 16-byte boundary."""
    v = 16 // {"f32": 4, "f64": 8, "c64": 8}[dt]
    used = 0
    for vj in (8, 4):
        for nt in (256, 512):
            for nvx in (8, 16, 32):
                for nvy in (8, 16, 32):
                    for k, (update, ma, mb) in enumerate(((0, 0, 0), (1, v - 1, 1))):
                        order = k ^ (nvx == 16)
                        rc, n = check_vtile(dt, size, perm, nt, nvx, nvy, order, update, ma, mb,
                                            vj)
                        assert rc == 0, (dt, size, perm, nt, nvx, nvy, vj, order, update, rc)
                        assert n in (0, np.prod(size))
                        used += n > 0
    assert used > 0, "no vector tile planned"


# Shapes a TMA tile can serve (every stride other than the unit one a
# multiple of 16 bytes, fused rank <= 5), with extents that are not
# multiples of the 128-byte boxes: the debug replay adds the TMA-tile forms
# for these, with both tensor maps checked against TMA's rules.
TTILE_SHAPES = [
    ("f32", [64, 48, 20], [2, 1, 0]),
    ("f32", [100, 36, 60], [1, 0, 2]),
    ("f64", [30, 18, 8], [2, 0, 1]),
    ("c64", [16, 5, 6, 10], [3, 1, 0, 2]),
    ("f32", [4, 8, 3, 5, 12], [4, 2, 0, 1, 3]),
    ("f32", [256, 256, 16], [2, 1, 0]),
    ("f32", [1000, 332], [1, 0]),
    ("f64", [258, 130], [1, 0]),
    ("f32", [8, 3, 4, 5, 4], [4, 2, 0, 3, 1]),  # fused rank 5
]


@pytest.mark.parametrize("dt,size,perm", TTILE_SHAPES)
def test_replay_ttile_shapes(dt, size, perm):
    assert "TMA" not in h.inspect_plan(dt, size, perm)  # not the default plan
    rc, n = check(dt, size, perm)
    assert rc == 0, (dt, size, perm, rc)
    assert n == np.prod(size)


def test_replay_ttile_outer_sizes():
    """Sub-tensors: outer extents keep the strides 16-byte multiples (and
    pass the reference's guard, which also wants out_outer[perm[i]] >=
    in_size[i])."""
    rc, n = check("f32", [40, 20, 12], [2, 0, 1], [44, 24, 12], [20, 40, 40])
    assert rc == 0 and n == 40 * 20 * 12
    rc, n = check("c64", [6, 10, 7], [1, 2, 0], [8, 10, 9], [12, 7, 10])
    assert rc == 0 and n == 6 * 10 * 7


def _random_ttile_case(seed):
    """A seeded problem a TMA tile can serve: no extent-1 dims, input dim 0
    and the output's leading dim in multiples of 16 bytes, so every stride
    other than the unit one is a 16-byte multiple (fusion can only merge such
    dims into longer ones)."""
    rng = np.random.default_rng(seed)
    dt = ["f32", "f64", "c64"][seed % 3]
    q = 4 if dt == "f32" else 2  # elements per 16 bytes
    rank = int(rng.integers(2, 6))
    while True:
        perm = [int(x) for x in rng.permutation(rank)]
        if perm[0] != 0:
            break
    size = [int(rng.integers(2, 9)) for _ in range(rank)]
    size[0] = q * int(rng.integers(1, 12))
    size[perm[0]] = q * int(rng.integers(1, 12))
    return dt, size, perm


def _tma_describable(dt, size, perm):
    """From the plan summary: fused rank <= 5, a true transpose, and every
    stride of A and B other than the unit one a multiple of 16 bytes."""
    import re
    d = h.inspect_plan(dt, size, perm)
    sa = [int(x) for x in re.search(r"strides A: (.*)", d).group(1).split()]
    sb = [int(x) for x in re.search(r"strides B: (.*)", d).group(1).split()]
    pm = [int(x) for x in re.search(r"perm \(output dim -> input dim\): (.*)", d).group(1).split()]
    esz = {"f32": 4, "f64": 8, "c64": 8}[dt]
    return (len(sa) <= 5 and pm[0] != 0 and all(v * esz % 16 == 0 for v in sa[1:]) and
            all(v * esz % 16 == 0 for k, v in enumerate(sb) if k != pm[0]))


@pytest.mark.parametrize("seed", range(24))
def test_replay_ttile_random(seed):
    dt, size, perm = _random_ttile_case(seed)
    assert _tma_describable(dt, size, perm), (dt, size, perm)
    rc, n = check(dt, size, perm)
    assert rc == 0, (dt, size, perm, rc)
    assert n == np.prod(size)
