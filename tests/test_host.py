"""Host planner (no device): index fusion and tile-shape invariants.

Fusion follows the reference rule (inc/hptt/param/parameter_trans.tcc:223-283):
neighbouring output dims that are consecutive, unpadded input dims fuse.
"""
import re

import numpy as np
import pytest

import hptt_b200 as h


def parse(text):
    out = {}
    out["rank"] = int(re.search(r"fused rank: (\d+)", text).group(1))
    out["n"] = [int(x) for x in re.search(r"extents \(input order\):([\d ]+)", text).group(1).split()]
    out["perm"] = [int(x) for x in re.search(r"perm \(output dim -> input dim\):([\d ]+)", text).group(1).split()]
    out["kind"] = "rows" if "kernel: rows" in text else "tile"
    m = re.search(r"TX=(\d+) TY=(\d+) LD=(\d+)", text)
    out["TX"], out["TY"], out["LD"] = (int(m.group(i)) for i in (1, 2, 3))
    m = re.search(r"tile W=(\d+)", text)
    out["W"] = int(m.group(1))
    out["tiles"] = int(re.search(r"tiles: (\d+)", text).group(1))
    out["smem"] = int(re.search(r"smem/CTA: (\d+)", text).group(1))
    return out


def test_fusion_shared_stride_one_example():
    # in_size {8,64,4,64,16,32}, perm {0,3,2,1,4,5}: dims 4,5 fuse
    p = parse(h.inspect_plan("c64", [8, 64, 4, 64, 16, 32], [0, 3, 2, 1, 4, 5]))
    assert p["rank"] == 5
    assert p["n"] == [8, 64, 4, 64, 512]
    assert p["perm"] == [0, 3, 2, 1, 4]


def test_fusion_none_possible():
    p = parse(h.inspect_plan("c64", [8, 64, 4, 64, 16, 32], [5, 2, 0, 4, 1, 3]))
    assert p["rank"] == 6


def test_fusion_drops_unit_dims():
    p = parse(h.inspect_plan("f32", [1, 906, 1, 906], [2, 3, 0, 1]))
    assert p["rank"] == 2 and p["n"] == [906, 906] and p["perm"] == [1, 0]


def test_identity_becomes_rank_one_copy():
    p = parse(h.inspect_plan("f64", [7, 9, 11], [0, 1, 2]))
    assert p["rank"] == 1 and p["n"] == [693] and p["kind"] == "rows"


def test_padding_blocks_fusion():
    # dims 0,1 adjacent and in order, but dim 0 is padded in A
    p = parse(h.inspect_plan("f32", [4, 5, 6], [2, 0, 1], in_outer_size=[8, 5, 6]))
    assert p["rank"] == 3
    p2 = parse(h.inspect_plan("f32", [4, 5, 6], [2, 0, 1]))
    assert p2["rank"] == 2 and p2["n"] == [20, 6]


def test_reference_guard_on_outer_sizes():
    # out_outer is indexed by output dim: out size = {5, 4}
    with pytest.raises(h.HpttError):
        h.inspect_plan("f32", [4, 5], [1, 0], out_outer_size=[4, 4])
    h.inspect_plan("f32", [4, 5], [1, 0], out_outer_size=[5, 4])


@pytest.mark.parametrize("seed", range(400))
def test_tile_invariants_random(seed):
    rng = np.random.default_rng(seed)
    rank = int(rng.integers(2, 7))
    dtype = ["f32", "f64", "c64", "c128"][seed % 4]
    size = [int(x) for x in np.exp(rng.uniform(0, np.log(300), rank)).astype(int) + 1]
    perm = [int(x) for x in rng.permutation(rank)]
    p = parse(h.inspect_plan(dtype, size, perm))
    assert p["tiles"] >= 1
    assert np.prod(p["n"]) == np.prod(size)
    if p["kind"] == "tile":
        assert p["W"] * p["TX"] <= 256 and p["W"] * p["TY"] <= 256
        assert p["LD"] >= p["W"] * p["TX"]
        assert p["smem"] <= 227 * 1024  # opt-in shared memory per CTA on sm_100


def test_bench_roofline_picks_the_dominant_kernel(monkeypatch, tmp_path):
    """bench.py's roofline: the kernel kind with the most device time, its
    algorithmic bytes over its back-to-back pass time, DRAM traffic from the
    committed per-kernel ratio."""
    import json
    import bench
    plans = [(None, 10**9, "tile", {}), (None, 2 * 10**9, "vtile", {}),
             (None, 10**9, "rows", {})]
    kind_ms = {"tile": 10.0, "vtile": 30.0, "rows": 5.0}   # summed over 5 steps
    monkeypatch.setattr(bench, "_peaks", lambda: (6000.0, "measured"))
    r = bench._roofline(plans, kind_ms, 5, {"k_vtile": 0.95, "k_tile": 1.01})
    assert r["kernel"] == "k_vtile"
    assert r["achieved"] == round(2e9 * 5 / 0.030 / 1e9, 1)
    assert r["frac"] == round(r["achieved"] / 6000.0, 4)
    assert r["traffic"] == int(2 * 10**9 * 0.95)
    assert r["share_of_device_time"] == round(30.0 / 45.0, 4)
    assert set(r["kernels"]) == {"k_tile", "k_vtile", "k_rows"}
    # the committed traffic file parses into per-kernel ratios
    t = bench._profiled_traffic()
    assert t is None or all(0.5 < v < 2.0 for v in t.values())


def test_bench_roofline_names_the_tma_kernels(monkeypatch):
    """A plan on either TMA-tile form is timed and named as its own kernel
    (no DRAM-traffic ratio is committed for them: traffic stays null)."""
    import bench
    assert {"tile", "vtile", "ttile", "ttile_pipe", "rows"} <= set(bench.KERNEL_OF_KIND)
    plans = [(None, 10**9, "ttile", {}), (None, 10**9, "ttile_pipe", {}),
             (None, 10**9, "tile", {})]
    kind_ms = {"ttile": 4.0, "ttile_pipe": 6.0, "tile": 3.0}
    monkeypatch.setattr(bench, "_peaks", lambda: (6000.0, "measured"))
    r = bench._roofline(plans, kind_ms, 2, {"k_tile": 1.0})
    assert r["kernel"] == "k_ttile_pipe"
    assert r["traffic"] is None
    assert set(r["kernels"]) == {"k_ttile", "k_ttile_pipe", "k_tile"}
