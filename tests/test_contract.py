"""Tensor contraction through the transposes (hptt_cuda_contract_*):
C[lc] = alpha * sum_K A[la] * B[lb] + beta * C[lc] as transpose - cuBLAS GEMM -
transpose, the output transpose applying alpha and beta.

CPU: label validation and status codes, the layout choice (which operands are
used in place, which transposes run), workspace sizes, the spec parser, and
the checker itself against a plain loop.
GPU: random contractions of every element type (batch labels, scalar
outputs, complex scalars, beta = 0 and beta != 0) within the checker's error
bound; outer products bit-exact against the element-type arithmetic (the GEMM
computes single products there, so every bit comes from the transposes);
graph replay bit-identical to direct launches; reset_data, set_coef, a
caller-supplied workspace and other streams.
"""
import itertools

import numpy as np
import pytest

import hptt_b200 as h
import oracle.contract as oc
from helpers import assert_same, seeded


# --------------------------------------------------------------------------
# CPU
# --------------------------------------------------------------------------
def _layout(dt, sa, la, sb, lb, lc):
    text, ws = h.inspect_contraction(dt, sa, la, sb, lb, lc)
    return text, ws


def test_in_place_gemm_layouts():
    # plain matrix products in every op combination: no transposes at all
    for la, lb, lc in [("ik", "kj", "ij"), ("ki", "kj", "ij"), ("ik", "jk", "ij"),
                       ("ki", "jk", "ij"), ("ik", "kj", "ji"), ("ki", "jk", "ji")]:
        ext = {"i": 5, "j": 7, "k": 3}
        text, ws = _layout("f32", [ext[x] for x in la], la, [ext[x] for x in lb], lb, lc)
        assert "A in place" in text and "B in place" in text, (la, lb, lc, text)
        assert "into C with alpha, beta" in text, text
        assert "transposes move 0 bytes" in text
        assert ws == 32 << 20  # the GEMM library's workspace only


def test_transposes_chosen_and_workspace():
    sa, sb = [4, 6, 5, 3], [3, 7, 6, 2]
    text, ws = _layout("f64", sa, "acid", sb, "dbcj", "abij")
    # a,i are M; b,j N; c,d K: A and B need transposes, C too
    assert "(transposed)" in text and "output transpose applies" in text
    na, nb, nc = np.prod(sa), np.prod(sb), 4 * 7 * 5 * 2
    align = lambda x: (x + 255) // 256 * 256  # noqa: E731
    assert ws == align(na * 8) + align(nb * 8) + align(nc * 8) + (32 << 20)


def test_batch_labels_and_scalar_output():
    text, _ = _layout("f32", [4, 5, 6], "bik", [6, 7, 4], "kjb", "ijb")
    assert "batch [" in text and "= 4" in text and "into C" in text
    text, _ = _layout("c128", [7, 9], "ab", [9, 7], "ba", "")
    assert "M [] = 1, N [] = 1" in text


def test_extent_one_labels_do_not_force_transposes():
    text, _ = _layout("f32", [1, 8, 1, 9], "xiyk", [9, 5], "kj", "ixjy")
    assert "A in place" in text and "B in place" in text and "into C" in text


@pytest.mark.parametrize("args,status", [
    (("f32", [3, 3], "ii", [3], "i", "i"), 15),        # repeated label
    (("f32", [3, 4], "ik", [5, 2], "kj", "ij"), 15),    # K extents differ
    (("f32", [3, 4], "ik", [4, 2], "kj", "i"), 15),     # j summed over B alone
    (("f32", [3, 4], "ik", [4, 2], "kj", "ijz"), 15),   # C label nowhere
    (("f32", [3, 4, 2], "ikz", [4, 2], "kj", "ij"), 15),  # z summed over A alone
    (("f32", [3, 0], "ik", [0, 2], "kj", "ij"), 4),     # zero extent
    (("q32", [3, 4], "ik", [4, 2], "kj", "ij"), 6),     # dtype
    (("f32", [2] * 9, "abcdefghi", [2], "a", "bcdefghi"), 2),  # rank 9
])
def test_rejects(args, status):
    if args[0] == "q32":
        lib = h.load_library()
        import ctypes
        st = lib.hptt_cuda_contract_inspect(9, 2, h._u32([3, 4]), h._i32([0, 1]), 2,
                                            h._u32([4, 2]), h._i32([1, 2]), 2,
                                            h._i32([0, 2]), None, 0, None)
        assert st == status
        return
    with pytest.raises(h.HpttError) as e:
        h.inspect_contraction(*args)
    assert e.value.status == status


def test_create_rejects_without_device_work():
    lib = h.load_library()
    import ctypes
    out = ctypes.c_void_p(0)
    one = h._scalar(1.0)
    st = lib.hptt_cuda_contract_create(0, 2, h._u32([3, 4]), h._i32([0, 1]), 2, h._u32([4, 2]),
                                       h._i32([1, 2]), 2, h._i32([0, 2]), one, one, 0, None,
                                       None, None, None, 0, ctypes.byref(out))
    assert st == 1 and not out.value
    assert lib.hptt_cuda_contract_create(0, 2, None, None, 0, None, None, 0, None, one, one, 0,
                                         1, 1, 1, None, 0, None) == 11
    for fn in ("exec", "sync", "destroy"):
        assert getattr(lib, "hptt_cuda_contract_" + fn)(None) == 11


def test_parse_spec():
    assert h.parse_spec("acid, dbcj -> abij") == (list("acid"), list("dbcj"), list("abij"))
    assert h.parse_spec("ab,ba->") == (list("ab"), list("ba"), [])
    with pytest.raises(ValueError):
        h.parse_spec("ab->a")


def _naive(sa, la, a, sb, lb, b, lc, c0, alpha, beta, upd):
    ext = dict(zip(la, sa))
    ext.update(zip(lb, sb))
    labels = list(dict.fromkeys(list(la) + list(lb) + list(lc)))
    A = a.reshape(sa, order="F")
    B = b.reshape(sb, order="F")
    sc = [ext[x] for x in lc]
    out = np.zeros(sc, dtype=np.complex128) if np.iscomplexobj(a) else np.zeros(sc)
    for idx in itertools.product(*[range(ext[x]) for x in labels]):
        v = dict(zip(labels, idx))
        out[tuple(v[x] for x in lc)] += A[tuple(v[x] for x in la)] * B[tuple(v[x] for x in lb)]
    out = alpha * out
    if upd:
        out = out + beta * c0.reshape(sc, order="F")
    return out.reshape(-1, order="F")


@pytest.mark.parametrize("name", ["f64", "c128"])
def test_checker_against_plain_loop(name):
    rng = np.random.default_rng(4)
    sa, la, sb, lb, lc = [3, 4, 2], "aib", [2, 4, 5], "bij", "jab"
    a = seeded(rng, 24, name)
    b = seeded(rng, 40, name)
    c0 = seeded(rng, 5 * 3 * 2, name)
    val, bound = oc.contract(name, sa, la, a, sb, lb, b, lc, c0, 0.5, -1.25)
    want = _naive(sa, la, a, sb, lb, b, lc, c0, 0.5, -1.25, True)
    oc.check(name, want.astype(oc.NP[name]), val, bound, "checker vs loop")
    # a planted error of a few ulp-scale bounds is caught
    bad = want.astype(oc.NP[name]).copy()
    bad[3] += 50 * bound[3]
    with pytest.raises(AssertionError):
        oc.check(name, bad, val, bound, "planted")


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


TD = {"f32": "float32", "f64": "float64", "c64": "complex64", "c128": "complex128"}


def _dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _random_contraction(rng, name, max_elems=40000):
    """Random labels: 0-2 each of M, N, K and batch (at least one of M, N or
    K), random orders in each tensor, extents 1-12."""
    while True:
        counts = [int(rng.integers(0, 3)) for _ in range(4)]
        if sum(counts[:3]) and sum(counts) <= 6 and counts[0] + counts[2] + counts[3] >= 1 \
                and counts[1] + counts[2] + counts[3] >= 1:
            break
    labels = iter("abcdefghijkl")
    M = [next(labels) for _ in range(counts[0])]
    N = [next(labels) for _ in range(counts[1])]
    K = [next(labels) for _ in range(counts[2])]
    Bt = [next(labels) for _ in range(counts[3])]
    ext = {x: int(rng.integers(1, 13)) for x in M + N + K + Bt}
    la = list(rng.permutation(M + K + Bt))
    lb = list(rng.permutation(K + N + Bt))
    lc = list(rng.permutation(M + N + Bt))
    for lst in (la, lb, lc):
        while lst and np.prod([ext[x] for x in lst]) > max_elems:
            big = max(lst, key=lambda x: ext[x])
            ext[big] = max(1, ext[big] // 2)
    return [ext[x] for x in la], la, [ext[x] for x in lb], lb, lc


def _scalars(rng, name, i):
    if i % 3 == 0:
        return 1.0, 0.0, False
    if name in ("c64", "c128") and i % 3 == 1:
        return (complex(rng.uniform(-2, 2), rng.uniform(-2, 2)),
                complex(rng.uniform(-2, 2), rng.uniform(-2, 2)), True)
    return float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2)), False


def _run_case(torch, name, sa, la, sb, lb, lc, alpha, beta, cs, seed, use_graph=True, execs=1):
    rng = np.random.default_rng(seed)
    a = seeded(rng, int(np.prod(sa)), name)
    b = seeded(rng, int(np.prod(sb)), name)
    sc = oc.out_size(sa, la, sb, lb, lc)
    c0 = seeded(rng, int(np.prod(sc)) if sc else 1, name)
    da, db, dc = _dev(torch, a), _dev(torch, b), _dev(torch, c0)
    plan = h.create_contraction(da, db, dc, sa, la, sb, lb, lc, alpha, beta, dtype=name,
                                complex_scalars=cs, use_graph=use_graph)
    want = c0
    for _ in range(execs):
        plan.exec()
        val, bound = oc.contract(name, sa, la, a, sb, lb, b, lc, want, alpha, beta, cs)
        want = val.astype(oc.NP[name])
    plan.sync()
    return plan, dc.cpu().numpy(), val, bound


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["f32", "f64", "c64", "c128"])
@pytest.mark.parametrize("seed", range(6))
def test_random_contractions(name, seed):
    torch = _torch()
    rng = np.random.default_rng(1000 * seed + len(name))
    for i in range(6):
        sa, la, sb, lb, lc = _random_contraction(rng, name)
        alpha, beta, cs = _scalars(rng, name, i)
        plan, got, val, bound = _run_case(torch, name, sa, la, sb, lb, lc, alpha, beta, cs,
                                          seed * 100 + i)
        what = f"{name} {la}{sa} x {lb}{sb} -> {lc} a={alpha} b={beta}\n{plan.describe()}"
        oc.check(name, got, val, bound, what)
        plan.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["f32", "f64", "c64", "c128"])
def test_named_layouts(name):
    """Every layout family: in-place GEMMs (N/T, swapped), all three
    transposes, batch labels, a scalar output, extent-1 labels."""
    torch = _torch()
    cases = [
        ([40, 24], "ik", [24, 36], "kj", "ij"),
        ([24, 40], "ki", [36, 24], "jk", "ji"),
        ([6, 5, 7, 4], "acid", [4, 9, 5, 3], "dbcj", "abij"),
        ([5, 6, 7], "bik", [7, 8, 5], "kjb", "ijb"),
        ([5, 6, 7], "bik", [7, 8, 5], "kjb", "jbi"),
        ([13, 17], "ab", [17, 13], "ba", ""),
        ([1, 8, 1, 9], "xiyk", [9, 5], "kj", "ixjy"),
        ([3, 4, 5, 6, 2], "abcde", [6, 5, 7, 2], "dcfe", "fbea"),
    ]
    for i, (sa, la, sb, lb, lc) in enumerate(cases):
        for alpha, beta, cs in [(1.0, 0.0, False), (-0.75, 1.5, False)] + (
                [(1.5 - 0.5j, 0.25 + 1j, True)] if name in ("c64", "c128") else []):
            plan, got, val, bound = _run_case(torch, name, sa, la, sb, lb, lc, alpha, beta, cs,
                                              7 + i)
            oc.check(name, got, val, bound, f"{name} {la},{lb}->{lc} a={alpha} b={beta}")
            plan.destroy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["f32", "f64"])
def test_outer_product_bit_exact(name):
    """K = 1: the GEMM computes single products fl(a*b); the output
    transpose then applies fl(fl(alpha*p) + fl(beta*c)).  Every bit of C is
    checked against that arithmetic in the element type."""
    torch = _torch()
    rng = np.random.default_rng(3)
    # C interleaves M and N labels, so neither GEMM output layout is C's
    sa, la, sb, lb, lc = [6, 1, 5], "iku", [7, 1, 3], "jkv", "ujvi"
    a = seeded(rng, 30, name)
    b = seeded(rng, 21, name)
    c0 = seeded(rng, 3 * 7 * 5 * 6, name)
    t = oc.NP[name]
    alpha, beta = t(-1.375), t(0.625)
    A = a.reshape(sa, order="F")[:, 0, :]
    B = b.reshape(sb, order="F")[:, 0, :]
    P = (A[:, :, None, None] * B[None, None, :, :]).astype(t)   # [i,u,j,v]
    P = np.transpose(P, (1, 2, 3, 0))                           # [u,j,v,i]
    C0 = c0.reshape([5, 7, 3, 6], order="F")
    want = (alpha * P).astype(t) + (beta * C0).astype(t)
    da, db, dc = _dev(torch, a), _dev(torch, b), _dev(torch, c0)
    plan = h.create_contraction(da, db, dc, sa, la, sb, lb, lc, float(alpha), float(beta),
                                dtype=name)
    assert "output transpose applies" in plan.describe()
    plan.exec()
    plan.sync()
    assert_same(dc.cpu().numpy(), want.reshape(-1, order="F").astype(t), name,
                "outer product")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["f32", "c128"])
def test_graph_replay_matches_direct(name):
    torch = _torch()
    sa, la, sb, lb, lc = [6, 5, 7, 4], "acid", [4, 9, 5, 3], "dbcj", "abij"
    outs = []
    for use_graph in (False, True):
        plan, got, val, bound = _run_case(torch, name, sa, la, sb, lb, lc, 0.5, 1.25, False, 9,
                                          use_graph=use_graph, execs=4)
        oc.check(name, got, val, bound, f"{name} graph={use_graph}")
        assert plan.info()["graph"] == (1 if use_graph else 0)
        outs.append(got)
        plan.destroy()
    assert_same(outs[1], outs[0], name, "graph vs direct")


@pytest.mark.gpu
def test_reset_data_set_coef_workspace_and_streams():
    torch = _torch()
    name = "f64"
    sa, la, sb, lb, lc = [6, 5, 7, 4], "acid", [4, 9, 5, 3], "dbcj", "abij"
    _, ws_bytes = h.inspect_contraction(name, sa, la, sb, lb, lc)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    rng = np.random.default_rng(12)
    sc = oc.out_size(sa, la, sb, lb, lc)
    bufs = []
    for _ in range(2):
        a = seeded(rng, int(np.prod(sa)), name)
        b = seeded(rng, int(np.prod(sb)), name)
        c0 = seeded(rng, int(np.prod(sc)), name)
        bufs.append((a, b, c0, _dev(torch, a), _dev(torch, b), _dev(torch, c0)))
    a, b, c0, da, db, dc = bufs[0]
    plan = h.create_contraction(da, db, dc, sa, la, sb, lb, lc, 2.0, 0.0, dtype=name,
                                workspace=ws)
    assert plan.info()["workspace_bytes"] == ws_bytes
    plan.exec()
    plan.exec()   # second exec captures and replays the graph
    plan.sync()
    val, bound = oc.contract(name, sa, la, a, sb, lb, b, lc, c0, 2.0, 0.0)
    oc.check(name, dc.cpu().numpy(), val, bound, "first buffers")
    a2, b2, c2, da2, db2, dc2 = bufs[1]
    plan.reset_data(da2, db2, dc2)
    plan.set_coef(-0.5, 3.0)
    s = torch.cuda.Stream()
    plan.exec_on(s)
    s.synchronize()
    val, bound = oc.contract(name, sa, la, a2, sb, lb, b2, lc, c2, -0.5, 3.0)
    oc.check(name, dc2.cpu().numpy(), val, bound, "after reset_data/set_coef")
    plan.destroy()
    with pytest.raises(h.HpttError) as e:
        h.create_contraction(da, db, dc, sa, la, sb, lb, lc, 1.0, 0.0, dtype=name,
                             workspace=ws[:1024])
    assert e.value.status == 10


@pytest.mark.gpu
def test_spec_helper():
    torch = _torch()
    name = "f32"
    rng = np.random.default_rng(21)
    sa, sb = [16, 12, 10], [10, 12, 9]
    a, b = seeded(rng, 16 * 12 * 10, name), seeded(rng, 10 * 12 * 9, name)
    c0 = seeded(rng, 9 * 16, name)
    da, db, dc = _dev(torch, a), _dev(torch, b), _dev(torch, c0)
    plan = h.contract("xyk,kyz->zx", da, db, dc, sa, sb, 1.0, 1.0)
    plan.exec()
    plan.sync()
    val, bound = oc.contract(name, sa, "xyk", a, sb, "kyz", b, "zx", c0, 1.0, 1.0)
    oc.check(name, dc.cpu().numpy(), val, bound, "spec helper")
