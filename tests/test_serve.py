"""Served form (hptt_cuda_server_*): requests admitted as they arrive against a
device-byte budget and run with continuous batching.

The central check: every request's result is the same alone and in the mix
-- bit-exact against its own plain exec and the oracle -- with many requests
in flight, small launches (max_batch) and a budget small enough that
admission has to wait; also through other buffers than the plan's, with the
same output submitted several times (serialised), and in per-call mode.
CPU tests cover the argument checks.
"""
import ctypes

import numpy as np
import pytest

import hptt_b200 as h
from helpers import assert_same, oracle_run, seeded
from test_batch import _mixed_cases, _setup, _torch


def test_server_argument_checks():
    lib = h.load_library()
    out = ctypes.c_void_p(0)
    for cfg in (h.ServeConfig(0, 4, 16, 0, 0), h.ServeConfig(1 << 30, 0, 16, 0, 0),
                h.ServeConfig(1 << 30, 4, 0, 0, 0)):
        assert lib.hptt_cuda_server_create(ctypes.byref(cfg), ctypes.byref(out)) == 4
    assert lib.hptt_cuda_server_create(None, ctypes.byref(out)) == 4
    assert lib.hptt_cuda_server_submit(None, None, None, None, None) == 11
    assert lib.hptt_cuda_server_wait(None, 1, 0.1) == 11
    assert lib.hptt_cuda_server_drain(None, 0.1) == 11
    assert lib.hptt_cuda_server_reset_stats(None) == 11
    assert lib.hptt_cuda_server_destroy(None) == 11


def _alone(c):
    return oracle_run(c["name"], c["size"], c["perm"], c["alpha"], c["beta"], c["a"], c["b0"],
                      complex_scalars=c["cs"])


@pytest.mark.gpu
@pytest.mark.parametrize("per_call", [False, True])
def test_alone_vs_mix(per_call):
    torch = _torch()
    cases = _setup(torch, _mixed_cases(31, 72), 31)
    # every plan also run alone through its own exec, on a copy of its B
    alone_gpu = []
    for c in cases:
        db = c["db"].clone()
        c["plan"].reset_data(c["da"], db)
        c["plan"].exec()
        c["plan"].sync()
        alone_gpu.append(db.cpu().numpy())
        c["plan"].reset_data(c["da"], c["db"])
    biggest = max(c["plan"].bytes for c in cases)
    srv = h.TransServer(budget_bytes=3 * biggest, max_inflight_launches=3, max_batch=7,
                        per_call=per_call)
    order = np.random.default_rng(3).permutation(len(cases))
    tickets = [srv.submit(cases[i]["plan"]) for i in order]
    srv.drain()
    for t in tickets:
        srv.wait(t, 1.0)
    st = srv.stats()
    assert st["completed"] == len(cases) and st["failed"] == 0
    assert st["peak_inflight_bytes"] <= 3 * biggest
    if not per_call:
        assert st["launches"] > 1
    srv.destroy()
    for c, g in zip(cases, alone_gpu):
        got = c["db"].cpu().numpy()
        what = f"{c['name']} {c['size']} {c['perm']} a={c['alpha']} b={c['beta']}"
        assert_same(got, g, c["name"], "mix vs alone exec: " + what)
        assert_same(got, _alone(c), c["name"], "mix vs oracle: " + what)


@pytest.mark.gpu
def test_other_buffers_and_repeated_outputs():
    """Requests on other buffers than the plan's, and the same output three
    times (each must see the previous one's result)."""
    torch = _torch()
    cases = _setup(torch, _mixed_cases(41, 16), 41)
    rng = np.random.default_rng(8)
    srv = h.TransServer(max_inflight_launches=4, max_batch=64)
    extra = []
    for c in cases:
        a2 = seeded(rng, c["a"].size, c["name"])
        b2 = seeded(rng, c["b0"].size, c["name"])
        da2 = torch.from_numpy(a2).cuda()
        db2 = torch.from_numpy(b2).cuda()
        extra.append((a2, b2, da2, db2))
    for c, (a2, b2, da2, db2) in zip(cases, extra):
        for _ in range(3):
            srv.submit(c["plan"])
        srv.submit(c["plan"], da2, db2)
    srv.drain()
    assert srv.stats()["completed"] == 4 * len(cases)
    srv.destroy()
    for c, (a2, b2, da2, db2) in zip(cases, extra):
        want = c["b0"]
        for _ in range(3):
            want = oracle_run(c["name"], c["size"], c["perm"], c["alpha"], c["beta"], c["a"],
                              want, complex_scalars=c["cs"])
        assert_same(c["db"].cpu().numpy(), want, c["name"], f"3x {c['name']} {c['size']}")
        want2 = oracle_run(c["name"], c["size"], c["perm"], c["alpha"], c["beta"], a2, b2,
                           complex_scalars=c["cs"])
        assert_same(db2.cpu().numpy(), want2, c["name"], f"other buffers {c['name']}")


@pytest.mark.gpu
def test_budget_rejects_oversize_and_poisson_smoke():
    torch = _torch()
    cases = _setup(torch, _mixed_cases(51, 12), 51)
    small = min(c["plan"].bytes for c in cases)
    big = max(cases, key=lambda c: c["plan"].bytes)
    srv = h.TransServer(budget_bytes=small // 2)
    with pytest.raises(h.HpttError) as e:
        srv.submit(big["plan"])
    assert e.value.status == 10
    srv.destroy()
    srv = h.TransServer(max_inflight_launches=4, max_batch=128)
    st = srv.run_poisson([c["plan"] for c in cases], rate=20000.0, seconds=0.2, seed=1)
    assert st["submitted"] > 1000 and st["completed"] == st["submitted"]
    assert st["failed"] == 0
    assert 0 < st["lat_p50_us"] <= st["lat_p99_us"] <= st["lat_p999_us"] <= st["lat_max_us"]
    # the scheduler thread's longest pass: some time, and no longer than the run
    assert 0 < st["sched_pass_max_us"] <= st["elapsed_s"] * 1e6 + 1e6
    srv.destroy()
