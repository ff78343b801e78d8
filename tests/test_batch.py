"""Batched form: many plans in one graph launch (hptt_cuda_batch_*).

Each entry of a batch must give exactly the bits its own plan's exec gives
(and the oracle gives), whatever else runs beside it: mixed element types,
ranks, permutations, sizes, scalars (real and complex), tile bodies (tile,
rows, vectorised and scalar rows), repeated execs (beta != 0 accumulates),
and refresh after reset_data / set_coef.  CPU tests cover the argument checks.
"""
import ctypes

import numpy as np
import pytest

import hptt_b200 as h
from helpers import assert_same, footprint, oracle_run, random_perm, seeded

NAMES = ["f32", "f64", "c64", "c128"]


def test_batch_rejects_bad_handles():
    lib = h.load_library()
    arr = (ctypes.c_void_p * 2)(None, None)
    out = ctypes.c_void_p(0)
    assert lib.hptt_cuda_batch_create(arr, 2, ctypes.byref(out)) == 11
    assert lib.hptt_cuda_batch_create(arr, 1, None) == 11
    assert lib.hptt_cuda_plan_exec_many(arr, 1, None) == 11
    for fn in (lib.hptt_cuda_batch_refresh, lib.hptt_cuda_batch_destroy):
        assert fn(None) == 11
    assert lib.hptt_cuda_batch_exec(None, None) == 11


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _tdt(torch, name):
    return {"f32": torch.float32, "f64": torch.float64, "c64": torch.complex64,
            "c128": torch.complex128}[name]


def _mixed_cases(seed, count, max_elems=60000):
    """Mixed transposes: every element type, ranks 2-6, random perms and
    extents, half alpha=1/beta=0, the rest random scalars (complex for half
    of the complex entries); some shared-stride-1 perms for the rows bodies."""
    rng = np.random.default_rng(seed)
    cases = []
    for i in range(count):
        name = NAMES[i % 4]
        rank = 2 + int(rng.integers(0, 5))
        size = [int(x) for x in np.exp(rng.uniform(0, np.log(40), rank)).astype(int) + 1]
        while int(np.prod(size)) > max_elems:
            size[int(np.argmax(size))] //= 2
        if i % 7 == 3:
            size[0] = 64 + int(rng.integers(0, 200))   # long shared stride-1 run
            while int(np.prod(size)) > max_elems:
                size[1 + int(np.argmax(size[1:]))] = max(1, size[1 + int(np.argmax(size[1:]))] // 2)
            perm = [0] + [1 + int(x) for x in rng.permutation(rank - 1)]
        else:
            perm = random_perm(rng, rank)
        if rng.random() < 0.5:
            al, be, cs = 1.0, 0.0, False
        elif name in ("c64", "c128") and rng.random() < 0.5:
            al = complex(rng.uniform(-2, 2), rng.uniform(-2, 2))
            be = complex(rng.uniform(-2, 2), rng.uniform(-2, 2))
            cs = True
        else:
            al, be, cs = float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2)), False
        cases.append(dict(name=name, size=size, perm=perm, alpha=al, beta=be, cs=cs))
    return cases


def _setup(torch, cases, seed, offset_elems=0):
    """Host inputs, device A/B per case, and one plan per case."""
    rng = np.random.default_rng(seed)
    out = []
    for c in cases:
        n_in, n_out = footprint(c["size"], c["perm"])
        a = seeded(rng, n_in, c["name"])
        b0 = seeded(rng, n_out, c["name"])
        t = _tdt(torch, c["name"])
        da = torch.empty(n_in + offset_elems, dtype=t, device="cuda")[offset_elems:]
        db = torch.empty(n_out + offset_elems, dtype=t, device="cuda")[offset_elems:]
        da.copy_(torch.from_numpy(a))
        db.copy_(torch.from_numpy(b0))
        p = h.create_plan(da, db, c["size"], c["perm"], c["alpha"], c["beta"], 0,
                          dtype=c["name"], complex_scalars=c["cs"])
        assert p is not None
        out.append(dict(c, a=a, b0=b0, da=da, db=db, plan=p))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1])
def test_batch_matches_each_plan_and_oracle(seed):
    torch = _torch()
    cases = _setup(torch, _mixed_cases(100 + seed, 64), seed)
    batch = h.create_batch([c["plan"] for c in cases])
    nbytes, items, kernels = batch.info()
    assert nbytes == sum(c["plan"].bytes for c in cases)
    assert items >= len(cases) and kernels >= 1
    batch.exec()
    torch.cuda.synchronize()
    got_batch = [c["db"].cpu().numpy() for c in cases]
    # the same plans one by one on fresh copies of B
    for c in cases:
        c["db"].copy_(torch.from_numpy(c["b0"]))
    for c in cases:
        c["plan"].exec()
    torch.cuda.synchronize()
    for c, gb in zip(cases, got_batch):
        what = f"{c['name']} {c['size']} {c['perm']} a={c['alpha']} b={c['beta']}"
        assert_same(gb, c["db"].cpu().numpy(), c["name"], "batch vs own exec: " + what)
        want = oracle_run(c["name"], c["size"], c["perm"], c["alpha"], c["beta"], c["a"],
                          c["b0"], complex_scalars=c["cs"])
        assert_same(gb, want, c["name"], "batch vs oracle: " + what)


@pytest.mark.gpu
def test_batch_repeated_exec_and_exec_many():
    """Two batch runs equal two sequential per-call runs (beta != 0
    entries read what the first run wrote)."""
    torch = _torch()
    cases = _setup(torch, _mixed_cases(7, 40), 7)
    batch = h.create_batch([c["plan"] for c in cases])
    s = torch.cuda.Stream()
    batch.exec(s)
    batch.exec(s)
    s.synchronize()
    got = [c["db"].cpu().numpy() for c in cases]
    for c in cases:
        c["db"].copy_(torch.from_numpy(c["b0"]))
    torch.cuda.synchronize()
    plans = [c["plan"] for c in cases]
    h.exec_many(plans, s)
    h.exec_many(plans, s)
    s.synchronize()
    for c, g in zip(cases, got):
        assert_same(g, c["db"].cpu().numpy(), c["name"], f"{c['name']} {c['size']} twice")


@pytest.mark.gpu
def test_batch_refresh_after_reset_data_and_set_coef():
    torch = _torch()
    cases = _setup(torch, _mixed_cases(11, 24), 11)
    batch = h.create_batch([c["plan"] for c in cases])
    batch.exec()
    torch.cuda.synchronize()
    # new buffers for every other entry (one of them misaligned by one
    # element, which moves vectorised rows entries to their scalar tile) and
    # new scalars for the rest
    rng = np.random.default_rng(5)
    for i, c in enumerate(cases):
        if i % 2 == 0:
            off = 1 if i % 4 == 0 else 0
            t = c["da"].dtype
            na = torch.empty(c["da"].numel() + off, dtype=t, device="cuda")[off:]
            nb = torch.empty(c["db"].numel() + off, dtype=t, device="cuda")[off:]
            c["a"] = seeded(rng, c["a"].size, c["name"])
            c["b0"] = seeded(rng, c["b0"].size, c["name"])
            na.copy_(torch.from_numpy(c["a"]))
            nb.copy_(torch.from_numpy(c["b0"]))
            c["da"], c["db"] = na, nb
            c["plan"].reset_data(na, nb)
        else:
            c["b0"] = c["db"].cpu().numpy()
            c["alpha"], c["beta"], c["cs"] = -0.75, 1.5, False
            c["plan"].set_coef(-0.75, 1.5)
    batch.refresh()
    batch.exec()
    torch.cuda.synchronize()
    for c in cases:
        want = oracle_run(c["name"], c["size"], c["perm"], c["alpha"], c["beta"], c["a"],
                          c["b0"], complex_scalars=c["cs"])
        assert_same(c["db"].cpu().numpy(), want, c["name"],
                    f"refresh {c['name']} {c['size']} {c['perm']}")


@pytest.mark.gpu
def test_empty_batch():
    _torch()
    b = h.create_batch([])
    assert b.info() == (0, 0, 0)
    b.exec()
    b.destroy()


@pytest.mark.gpu
def test_batch_benchmark_sizes_against_oracle():
    """A quarter of the benchmark's 4096-transpose mixed workload (every
    fourth entry: 1024 transposes of 4 KB - 16 MB each, all four element
    types, ranks 2-6, half alpha=1/beta=0, complex scalars for complex types)
    plus one entry of each tile body that quarter misses, at its own sizes and
    with the shipped tuned tiles, run as one batch: every entry compared with
    the oracle bit for bit, and the batch uses as many group kernels (tile
    bodies) as the whole workload does."""
    import os
    import oracle
    from hptt_b200.workloads import batch_cases
    torch = _torch()
    path = os.path.join(os.path.dirname(h.__file__), "tune", "b200.cache")
    h.tune_cache_clear()
    if os.path.exists(path):
        h.tune_cache_load(path)
    try:
        allc = batch_cases()
        # group kernels of the whole workload: plans only record pointers, so
        # one scratch buffer of the largest footprint stands in for every
        # tensor (nothing is launched on it)
        biggest = max(int(np.prod(c["in_size"])) * {"f32": 4, "f64": 8, "c64": 8,
                                                   "c128": 16}[c["dtype"]] for c in allc)
        scratch = torch.empty(biggest, dtype=torch.uint8, device="cuda")
        dry = [h.create_plan(scratch, scratch, c["in_size"], c["perm"], c["alpha"], c["beta"],
                             0, dtype=c["dtype"]) for c in allc]
        full_kernels = h.create_batch(dry).info()[2]
        # every fourth entry, plus the first entry of every body that subset
        # misses (found by growing the batch one entry at a time)
        chosen = list(range(0, len(allc), 4))
        have = h.create_batch([dry[i] for i in chosen]).info()[2]
        for i in range(len(allc)):
            if have == full_kernels:
                break
            if i % 4 == 0:
                continue
            k = h.create_batch([dry[j] for j in chosen] + [dry[i]]).info()[2]
            if k > have:
                chosen.append(i)
                have = k
        del dry
        cases = [allc[i] for i in sorted(chosen)]
        g = torch.Generator(device="cuda").manual_seed(44)
        ents = []
        for c in cases:
            n = int(np.prod(c["in_size"]))
            t = _tdt(torch, c["dtype"])
            if c["dtype"] in ("c64", "c128"):
                rt = torch.float32 if c["dtype"] == "c64" else torch.float64
                da = torch.view_as_complex(torch.rand(n, 2, generator=g, device="cuda", dtype=rt) * 2 - 1)
                db = torch.view_as_complex(torch.rand(n, 2, generator=g, device="cuda", dtype=rt) * 2 - 1)
            else:
                da = torch.rand(n, generator=g, device="cuda", dtype=t) * 2 - 1
                db = torch.rand(n, generator=g, device="cuda", dtype=t) * 2 - 1
            b0 = db.cpu().numpy()
            p = h.create_plan(da, db, c["in_size"], c["perm"], c["alpha"], c["beta"], 0,
                              dtype=c["dtype"])
            assert p is not None
            ents.append((c, da, db, b0, p))
        batch = h.create_batch([e[4] for e in ents])
        nbytes, items, kernels = batch.info()
        assert kernels == full_kernels, (kernels, full_kernels)
        batch.exec()
        torch.cuda.synchronize()
        for c, da, db, b0, p in ents:
            a = oracle.aligned_empty(da.numel(), oracle.NP_DTYPES[c["dtype"]])
            a[:] = da.cpu().numpy()
            b0a = oracle.aligned_empty(b0.size, b0.dtype)
            b0a[:] = b0
            cs = isinstance(c["alpha"], complex) or isinstance(c["beta"], complex)
            want = oracle_run(c["dtype"], c["in_size"], c["perm"], c["alpha"], c["beta"], a,
                              b0a, complex_scalars=cs)
            assert_same(db.cpu().numpy(), want, c["dtype"],
                        f"batch entry {c['dtype']} {c['in_size']} {c['perm']} "
                        f"a={c['alpha']} b={c['beta']}")
        batch.destroy()
    finally:
        h.tune_cache_clear()
