#!/usr/bin/env python3
"""Benchmark: B = alpha * A(perm) + beta * B on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sweep|plain|hard] [--tune-cache PATH | --no-tune-cache]
                    [--case I]

Default workload ("sweep"): the plain permutation sweep -- 48 seeded cases over
ranks 2-6 in f32/f64, random non-identity permutations, extents log-uniform in
[4, 4096] rescaled to ~200 MB per tensor, each run with alpha=1, beta=0 and
with alpha=2.3, beta=4.2.  One step = all 96 transposes, every tensor resident
in HBM (19.2 GB); tensors are larger than L2, so no L2 flush is needed.

value     = algorithmic bytes of all transposes of all ranks / max-over-ranks
            device time (bytes = 2*N*sizeof(T), + N*sizeof(T) when B is read)
e2e       = the same metric through the C ABI with host buffers: every step
            copies A (and B when it is read) from pinned host memory, runs
            exec, and copies B back, all inside the timed region
roofline  = the dominant kernel's achieved bandwidth over the measured HBM
            copy peak (MEASURED_PEAKS.json); traffic = its DRAM bytes per
            launch from the committed ncu summary (profiles/traffic.json)
tiles     = from the shipped autotune cache (hptt_b200/tune/b200.cache, made
            on a B200 by `python -m hptt_b200.tune_sweep`); a shape it does
            not hold uses the planner's heuristic (--no-tune-cache: always)
cpu_baseline = the reference's own CPU code (oracle/_ref, built from the
            reference sources) on a bounded sample of the same workload, all
            host threads: its plan where that plan is correct for the shape,
            else its naive RefTrans, labelled.
plain     = config 1 (f32 {256,256,256}, perm {2,1,0}, alpha 2.3, beta 4.2):
            device GB/s with L2 flushed before every timed launch, roofline,
            e2e, and the reference plan at 1 thread and at all host threads
hard      = config 3 (c64/c128 rank-6 hard layouts, complex scalars): device
            GB/s, roofline, e2e, the reference's naive transpose on the host
            (complex scalars are not expressible through the reference API)

served   = the served form: Poisson arrivals over the same 4096 plans at
            10k-500k requests/s (2 s windows by default, --serve-seconds 60
            for the full run), 32 GB admission budget, continuous batching vs
            the plain per-call loop: throughput and p50/p99/p99.9 latency
            (--no-served skips it)
batched  = the batched form on the 4096-transpose mixed workload: one graph
            launch per run vs one plain exec per transpose (C loop, and the
            Python loop), same plans and buffers (--no-batched skips it)

N > 1 (torchrun): every rank runs the whole workload on its own GPU
(independent transposes; no collective on the data path), scaling "weak".
`--impl reference` times only the reference's CPU implementation (rank 0):
every step the whole workload (all 96 sweep transposes), all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GB/s & % HBM peak per transpose; batched req/s + p99 vs plain per-call exec"
DEFAULT_TUNE_CACHE = os.path.join(ROOT, "hptt_b200", "tune", "b200.cache")


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _workload(name):
    from hptt_b200 import workloads as w
    if name == "sweep":
        cases = []
        for c in w.sweep_cases():
            cases.append(dict(c, alpha=1.0, beta=0.0))
            cases.append(dict(c, alpha=2.3, beta=4.2))
        return cases, "permutation sweep: 48 cases (ranks 2-6, f32/f64, ~200 MB/tensor) x {a=1,b=0; a=2.3,b=4.2}"
    if name == "plain":
        return [w.plain_single()], "f32 {256,256,256} perm {2,1,0} a=2.3 b=4.2"
    if name == "hard":
        return w.hard_cases(), "c64/c128 rank-6 hard layouts, complex scalars"
    raise SystemExit(f"unknown workload {name}")


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def max_over_ranks(x: float, dist, world: int, device: str = "cuda") -> float:
    """The largest of every rank's x (x itself on one rank).  Every rank must
    call it at the same point: it is one all-reduce."""
    if world <= 1 or dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])


def aggregate_gbs(bytes_per_rank: int, world: int, max_ms: float) -> float:
    """Whole-job throughput: the bytes all ranks moved over the slowest rank's
    time (every rank runs the same workload: replicas, weak scaling)."""
    return bytes_per_rank * world / (max_ms / 1e3) / 1e9


def _tdtype(torch, name):
    return {"f32": torch.float32, "f64": torch.float64, "c64": torch.complex64,
            "c128": torch.complex128}[name]


def _make_plans(cases, rank):
    """Resident buffers (one A and one B per distinct tensor shape) and one
    plan per transpose; seeded uniform[-1, 1] data made on the device."""
    import torch
    import hptt_b200 as h
    from hptt_b200.workloads import algorithmic_bytes
    bufs = {}
    plans = []
    g = torch.Generator(device="cuda").manual_seed(1234 + rank)
    for c in cases:
        key = (c["dtype"], tuple(c["in_size"]), tuple(c["perm"]))
        if key not in bufs:
            n = int(np.prod(c["in_size"]))
            t = _tdtype(torch, c["dtype"])
            if c["dtype"] in ("c64", "c128"):
                rt = torch.float32 if c["dtype"] == "c64" else torch.float64
                a = torch.view_as_complex((torch.rand(n, 2, generator=g, device="cuda", dtype=rt) * 2 - 1).contiguous())
                b = torch.view_as_complex((torch.rand(n, 2, generator=g, device="cuda", dtype=rt) * 2 - 1).contiguous())
            else:
                a = torch.rand(n, generator=g, device="cuda", dtype=t) * 2 - 1
                b = torch.rand(n, generator=g, device="cuda", dtype=t) * 2 - 1
            bufs[key] = (a, b)
        a, b = bufs[key]
        p = h.create_plan(a, b, c["in_size"], c["perm"], c["alpha"], c["beta"], 0,
                          dtype=c["dtype"])
        assert p is not None
        d = p.describe()
        kind = ("rows" if "kernel: rows" in d else
                "vtile" if "kernel: vector tile" in d else
                ("ttile_pipe" if "persistent" in d else "ttile") if "kernel: TMA tile" in d else
                "tile")
        plans.append((p, algorithmic_bytes(c), kind, c))
    torch.cuda.synchronize()
    return plans, bufs


def _timed_steps(plans, steps, warmup, stream, dist, world, flush=None):
    """Warm-up, then the timed passes.  Pass 1 brackets `steps` steps (every
    transpose once per step, launched back to back as a caller issues them;
    consecutive launches overlap their launch and CTA start-up, see
    kernels.cu) with one CUDA event pair: the step time.  Pass 2, for the
    roofline, runs `steps` steps of each kernel kind alone -- that kind's
    transposes, in workload order, back to back -- between one event pair
    per kind: each kernel's average launch duration in a stream of its own
    launches.  Returns the max-over-ranks time of pass 1 (ms), the per-kind
    times of pass 2 (ms, summed over the steps) and the clock samples.
    flush: an L2 flush before every launch, outside per-launch event pairs;
    the step time and the kind times are then sums of per-launch times."""
    import torch
    sptr = stream.cuda_stream
    kinds = sorted({k for _, _, k, _ in plans})

    def step(record=None, only=None):
        for i, (p, _, kind, _) in enumerate(plans):
            if only is not None and kind != only:
                continue
            if flush is not None:
                flush()
            if record is not None:
                record[i][0].record(stream)
            p.exec_on(sptr)
            if record is not None:
                record[i][1].record(stream)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    kind_ms = {}
    if flush is None:
        t0, t1 = ev(), ev()
        torch.cuda.synchronize()
        t0.record(stream)
        for k in range(steps):
            step()
        t1.record(stream)
        torch.cuda.synchronize()
        elapsed_ms = t0.elapsed_time(t1)
        for kind in kinds:
            k0, k1 = ev(), ev()
            k0.record(stream)
            for k in range(steps):
                step(only=kind)
            k1.record(stream)
            torch.cuda.synchronize()
            kind_ms[kind] = k0.elapsed_time(k1)
    else:
        rec = [[(ev(), ev()) for _ in plans] for _ in range(steps)]
        for k in range(steps):
            step(rec[k])
        torch.cuda.synchronize()
        per_launch = [sum(rec[k][i][0].elapsed_time(rec[k][i][1]) for k in range(steps))
                      for i in range(len(plans))]
        for (_, _, kind, _), ms in zip(plans, per_launch):
            kind_ms[kind] = kind_ms.get(kind, 0.0) + ms
        elapsed_ms = sum(per_launch)
    clocks = sampler.stop()
    elapsed_ms = max_over_ranks(elapsed_ms, dist, world)
    return elapsed_ms, kind_ms, clocks


KERNEL_OF_KIND = {"tile": "k_tile", "vtile": "k_vtile", "ttile": "k_ttile",
                  "ttile_pipe": "k_ttile_pipe", "rows": "k_rows"}


def _roofline(plans, kind_ms, steps, traffic=None):
    """The dominant kernel (most device time): its algorithmic bytes per
    launch over its average launch duration (kind_ms from _timed_steps),
    against the measured peak.  traffic: DRAM bytes per algorithmic byte of
    that kernel from the committed single-launch captures, or None."""
    by_kind = {}
    for p, bb, kind, _ in plans:
        d = by_kind.setdefault(kind, [0, 0])
        d[0] += bb * steps
        d[1] += steps
    device_ms = sum(kind_ms.values())
    dom = max(kind_ms, key=lambda k: kind_ms[k])
    dom_ms = kind_ms[dom]
    dom_bytes, dom_launches = by_kind[dom]
    peak, peak_kind = _peaks()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    per_launch = int(dom_bytes // max(1, dom_launches))
    ratio = (traffic or {}).get(KERNEL_OF_KIND[dom])
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": int(per_launch * ratio) if ratio else None,
            "kernel": KERNEL_OF_KIND[dom],
            "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
                            if peak_kind == "measured" else
                            "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"),
            "launches": dom_launches,
            "algorithmic_bytes_per_launch": per_launch,
            "share_of_device_time": round(dom_ms / device_ms, 4),
            "timing": "that kernel's transposes alone, back to back, one event pair per pass",
            "kernels": {KERNEL_OF_KIND[k]: {"ms_per_step": round(kind_ms[k] / steps, 4),
                                            "GB/s": round(by_kind[k][0] / (kind_ms[k] / 1e3) / 1e9, 1),
                                            "launches_per_step": by_kind[k][1] // steps}
                        for k in kind_ms}}


def _l2_flush():
    """A callable that overwrites a 256 MB device buffer (twice the L2)."""
    import torch
    junk = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    return lambda: junk.fill_(1)


def run_section(args, name, stream):
    """One more workload measured the way the sweep is: device GB/s with the
    dominant kernel's roofline, the end-to-end figure through the C ABI with
    host buffers, and the reference's CPU code on the same cases.  The plain
    single transpose (64 MB tensors: A and B together about the size of L2)
    flushes L2 before every timed launch; the hard layouts (~256 MB tensors)
    need no flush."""
    cases, desc = _workload(name)
    plans, bufs = _make_plans(cases, 0)
    flush = _l2_flush() if name == "plain" else None
    steps = 50 if name == "plain" else 20
    ms, kind_ms, clocks = _timed_steps(plans, steps, 3, stream, None, 1, flush=flush)
    bytes_step = sum(bb for _, bb, _, _ in plans)
    peak, _ = _peaks()
    value = bytes_step * steps / (ms / 1e3) / 1e9
    out = {"workload": desc, "transposes_per_step": len(plans), "bytes_per_step": bytes_step,
           "steps": steps, "value": round(value, 1), "unit": "GB/s",
           "ms_per_step": round(ms / steps, 4), "hbm_frac": round(value / peak, 4),
           "l2": ("L2 flushed (256 MB write) before every timed launch; per-launch events"
                  if flush is not None else "inputs larger than L2 (no flush)"),
           "roofline": _roofline(plans, kind_ms, steps),
           "e2e": (run_e2e(args, plans, bufs, stream, e2e_steps=max(args.e2e_steps, 24 // len(plans)))
                   if args.e2e_steps > 0 else None),
           "clocks": clocks}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = (cpu_baseline_plain() if name == "plain"
                               else cpu_baseline_sample(cases, budget_s=args.cpu_budget))
    for p, _, _, _ in plans:
        p.destroy()
    del bufs
    return out


def run_ours(args, rank, world, dist):
    import torch
    import hptt_b200 as h

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    cases, desc = _workload(args.workload)
    if args.case is not None:
        cases = [cases[args.case]]
        desc += f" -- transpose {args.case} only"
    stream = torch.cuda.current_stream()
    tiles = "planner heuristic"
    if not args.no_tune_cache and args.tune_cache and os.path.exists(args.tune_cache):
        h.tune_cache_load(args.tune_cache)
        tiles = (f"autotune cache {os.path.relpath(args.tune_cache, ROOT)} "
                 f"({h.tune_cache_size()} entries; heuristic on a miss)")
    if args.batched_only or args.served_only:
        # the batched or served form alone (profiling; --batch-count,
        # --serve-rates, --serve-seconds)
        pool, pool_buffers = _batch_pool(args)
        out = {"tiles": tiles}
        if args.batched_only:
            out["batched"] = run_batched(args, stream, pool)
        if args.served_only:
            out["served"] = run_served(args, pool)
        del pool, pool_buffers
        return out

    plans, bufs = _make_plans(cases, rank)
    flush = _l2_flush() if args.workload == "plain" else None
    elapsed_ms, kind_ms, clocks = _timed_steps(plans, args.steps, args.warmup, stream,
                                               dist, world, flush=flush)
    device_ms = sum(kind_ms.values())
    bytes_step = sum(bb for _, bb, _, _ in plans)
    value = aggregate_gbs(bytes_step * args.steps, world, elapsed_ms)
    ms_per_step = elapsed_ms / args.steps
    peak, _ = _peaks()
    # DRAM traffic per launch: the committed single-launch ncu captures of
    # sample sweep cases (profiles/traffic.json), as a ratio to algorithmic
    # bytes per kernel
    ratio = _profiled_traffic() if args.workload == "sweep" and args.case is None else None
    roofline = _roofline(plans, kind_ms, args.steps, ratio)

    e2e = run_e2e(args, plans, bufs, stream, dist, world) if args.e2e_steps > 0 else None
    gpu_launches = sum(p.launches for p, _, _, _ in plans) * args.steps
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(cases, budget_s=args.cpu_budget)
    for p, _, _, _ in plans:
        p.destroy()
    del bufs
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    # the batched and served forms and the other configurations are measured
    # on one GPU (N > 1 runs replicas of the sweep only)
    batched = served = contraction = plain = hard = None
    single = world == 1 and args.case is None and args.workload == "sweep"
    if single and not args.no_sections:
        plain = run_section(args, "plain", stream)
        hard = run_section(args, "hard", stream)
        torch.cuda.empty_cache()
    if single and not (args.no_batched and args.no_served):
        pool, pool_buffers = _batch_pool(args)
        if not args.no_batched:
            batched = run_batched(args, stream, pool)
        if not args.no_served:
            served = run_served(args, pool)
        del pool, pool_buffers
    if single and not args.no_contraction:
        contraction = run_contractions(args)

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.workload == "sweep" else cases[0]["dtype"],
        "data": "synthetic (seeded uniform[-1,1]; shapes from the workload generator)",
        "config": {"workload": desc, "transposes_per_step": len(plans),
                   "bytes_per_step": bytes_step,
                   "l2": ("L2 flushed (256 MB write) before every timed launch"
                          if flush is not None else "inputs larger than L2 (no flush)"),
                   "tiles": tiles,
                   "parallelism": f"replicas x{world}"},
        "hbm_frac": round(value / world / peak, 4),
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "plain": plain,
        "hard": hard,
        "batched": batched,
        "served": served,
        "contraction": contraction,
        "kernel_ms_per_step": round(device_ms / args.steps, 4),
    }
    return out


def _profiled_traffic():
    """DRAM bytes (read + write) per algorithmic byte of each kernel, from the
    committed single-launch ncu captures of sample sweep cases
    (profiles/traffic.json; the captures and their command are in
    profiles/traffic_sweep_cases.md)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        return {k: float(v["dram_per_algorithmic_byte"]) for k, v in d["kernels"].items()}
    except Exception:
        return None


def run_e2e(args, plans, bufs, stream, dist=None, world=1, e2e_steps=None):
    """Same workload through the C ABI with host buffers, copies timed.

    Every transpose copies its A (and B when B is read) from pinned host
    memory into a device staging pair, points its plan there (reset_data),
    runs exec, and copies B back to pinned host memory.  Transposes rotate
    over three streams with one staging pair each, so one transpose's
    host->device copy overlaps the previous ones' kernels and device->host
    copies (PCIe is full duplex) without waiting for a staging pair; the
    rotation continues across steps, so with one transpose per step (the
    plain workload) a step's upload overlaps the previous step's download."""
    import torch
    host = {}
    for key, (a, b) in bufs.items():
        ha = torch.empty_like(a, device="cpu").pin_memory()
        hb = torch.empty_like(b, device="cpu").pin_memory()
        ha.copy_(a.cpu())
        hb.copy_(b.cpu())
        host[key] = (ha, hb)
    max_bytes = max(a.numel() * a.element_size() for a, _ in bufs.values())
    streams = [torch.cuda.Stream() for _ in range(3)]
    stage = [(torch.empty(max_bytes, dtype=torch.uint8, device="cuda"),
              torch.empty(max_bytes, dtype=torch.uint8, device="cuda"),
              torch.empty(max_bytes, dtype=torch.uint8).pin_memory()) for _ in streams]
    h2d = d2h = 0
    work = []
    for p, bb, kind, c in plans:
        key = (c["dtype"], tuple(c["in_size"]), tuple(c["perm"]))
        a, _ = bufs[key]
        nbytes = a.numel() * a.element_size()
        reads_b = bb > 2 * nbytes
        h2d += nbytes * (2 if reads_b else 1)
        d2h += nbytes
        work.append((p, key, nbytes, reads_b, a.dtype))

    issued = [0]  # transposes issued so far: consecutive ones, also across
                  # steps, go to different streams and staging pairs

    def step():
        for p, key, nbytes, reads_b, dt in work:
            i = issued[0]
            issued[0] += 1
            s = streams[i % len(streams)]
            sa, sb, hout = stage[i % len(streams)]
            ha, hb = host[key]
            da = sa[:nbytes].view(dt)
            db = sb[:nbytes].view(dt)
            with torch.cuda.stream(s):
                da.copy_(ha, non_blocking=True)
                if reads_b:
                    db.copy_(hb, non_blocking=True)
                p.reset_data(da, db)
                p.exec_on(s.cuda_stream)
                hout[:nbytes].view(dt).copy_(db, non_blocking=True)

    def timed(nsteps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in streams:
            s.wait_event(e0)
        for _ in range(nsteps):
            step()
        for s in streams:
            ev = torch.cuda.Event()
            ev.record(s)
            stream.wait_event(ev)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    nsteps = e2e_steps or args.e2e_steps
    timed(1)  # warm-up
    ms = timed(nsteps)
    ms = max_over_ranks(ms, dist, world)
    total = sum(bb for _, bb, _, _ in plans) * nsteps
    return {"value": round(aggregate_gbs(total, world, ms), 2), "unit": "GB/s",
            "h2d_bytes_per_step": h2d * world, "d2h_bytes_per_step": d2h * world,
            "steps": nsteps, "ms_per_step": round(ms / nsteps, 3),
            "api": "TransPlan.reset_data + exec_on (C ABI) with pinned host<->device "
                   "copies, three streams"}


def _batch_pool(args):
    """The mixed workload's plans and resident buffers: 4096 transposes
    (f32/f64/c64/c128, ranks 2-6, 4 KB - 16 MB per tensor, half alpha=1/
    beta=0, complex scalars for complex types), tiles from the autotune
    cache.  16.6 GB of tensors, far larger than L2 (no flush needed)."""
    import torch
    import hptt_b200 as h
    from hptt_b200 import workloads as w

    cases = w.batch_cases(count=args.batch_count)
    g = torch.Generator(device="cuda").manual_seed(77)
    plans, keep = [], []
    for c in cases:
        n = int(np.prod(c["in_size"]))
        t = _tdtype(torch, c["dtype"])
        if c["dtype"] in ("c64", "c128"):
            rt = torch.float32 if c["dtype"] == "c64" else torch.float64
            a = torch.view_as_complex(torch.rand(n, 2, generator=g, device="cuda", dtype=rt) * 2 - 1)
            b = torch.view_as_complex(torch.rand(n, 2, generator=g, device="cuda", dtype=rt) * 2 - 1)
        else:
            a = torch.rand(n, generator=g, device="cuda", dtype=t) * 2 - 1
            b = torch.rand(n, generator=g, device="cuda", dtype=t) * 2 - 1
        p = h.create_plan(a, b, c["in_size"], c["perm"], c["alpha"], c["beta"], 0,
                          dtype=c["dtype"])
        assert p is not None
        plans.append(p)
        keep.append((a, b))
    return plans, keep


def run_batched(args, stream, plans):
    """The batched form on the mixed workload pool.  One run = the whole
    set, timed three ways on the same plans and buffers:
      batch     one graph launch (hptt_cuda_batch_exec)
      per_call  one plain exec per transpose from a C loop
                (hptt_cuda_plan_exec_many)
      per_call_python  one TransPlan.exec_on per transpose from Python"""
    import torch
    import hptt_b200 as h

    batch = h.create_batch(plans)
    nbytes, items, kernels = batch.info()
    sptr = stream.cuda_stream

    def timed(fn, reps):
        fn()
        fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    reps = max(3, args.batch_reps)
    batch_ms = timed(lambda: batch.exec(sptr), reps)
    call_ms = timed(lambda: h.exec_many(plans, sptr), reps)

    def py_loop():
        for p in plans:
            p.exec_on(sptr)
    py_ms = timed(py_loop, 3)
    n = len(plans)
    out = {
        "workload": f"{n} mixed transposes (f32/f64/c64/c128, ranks 2-6, 4 KB-16 MB per "
                    "tensor, half alpha=1/beta=0, complex scalars for complex types)",
        "transposes": n,
        "bytes_per_run": nbytes, "work_items": items, "kernels_per_run": kernels,
        "batch": {"ms": round(batch_ms, 4), "GB/s": round(nbytes / batch_ms / 1e6, 1),
                  "transposes_per_s": round(n / batch_ms * 1e3, 1), "launches": 1,
                  "api": "hptt_cuda_batch_exec (one CUDA graph launch)"},
        "per_call": {"ms": round(call_ms, 4), "GB/s": round(nbytes / call_ms / 1e6, 1),
                     "transposes_per_s": round(n / call_ms * 1e3, 1), "launches": n,
                     "api": "hptt_cuda_plan_exec_many (C loop of plain execs)"},
        "per_call_python": {"ms": round(py_ms, 4), "GB/s": round(nbytes / py_ms / 1e6, 1),
                            "api": "TransPlan.exec_on per transpose from Python"},
        "speedup_vs_per_call": round(call_ms / batch_ms, 3),
        "speedup_vs_per_call_python": round(py_ms / batch_ms, 3),
        "reps": reps,
    }
    batch.destroy()
    return out


def run_served(args, plans):
    """The served form: open-loop Poisson arrivals over the mixed pool (each
    request a uniformly drawn plan on its resident buffers) at each rate for
    --serve-seconds, admission budget 32 GB; continuous batching vs the plain
    per-call loop (one exec per request, in arrival order, one stream) on the
    same GPU.  Arrivals come from the library's native generator
    (hptt_cuda_server_run_poisson).  Each rate is preceded by an untimed
    0.25 s run at that rate."""
    import hptt_b200 as h

    budget = 32 << 30
    rates = [float(r) for r in args.serve_rates.split(",")]
    keys = ("submitted", "completed", "launches", "mean_batch", "throughput_rps", "gbs",
            "lat_p50_us", "lat_p99_us", "lat_p999_us", "lat_max_us", "peak_inflight_bytes",
            "peak_pending", "sched_pass_max_us")
    out = {"budget_bytes": budget, "seconds_per_rate": args.serve_seconds,
           "pool": len(plans), "rates": []}
    for mode in ("batched", "per_call"):
        srv = h.TransServer(budget_bytes=budget,
                            max_inflight_launches=4 if mode == "batched" else 1024,
                            max_batch=1024, per_call=(mode == "per_call"))
        for k, rate in enumerate(rates):
            # a short untimed run at the same rate first (staging growth and
            # first launches of new batch sizes stay out of the numbers)
            srv.run_poisson(plans, rate=rate, seconds=0.25, seed=2000 + k, drain_timeout=600.0)
            srv.reset_stats()
            st = srv.run_poisson(plans, rate=rate, seconds=args.serve_seconds, seed=1000 + k,
                                 drain_timeout=600.0)
            row = next((r for r in out["rates"] if r["rate"] == rate), None)
            if row is None:
                row = {"rate": rate}
                out["rates"].append(row)
            row[mode] = {kk: (round(st[kk], 2) if isinstance(st[kk], float) else st[kk])
                         for kk in keys}
        srv.destroy()
    return out


def run_contractions(args):
    """Tensor contractions through the transposes (hptt_cuda_contract_*):
    seeded synthetic TTGT workloads (workloads.contraction_cases), each timed
    three ways on the same device buffers with CUDA events:
      ours       one contraction exec (graph replay: operand transposes, one
                 strided-batched cuBLAS GEMM, output transpose with alpha/beta)
      gemm_only  a contraction of the same m, n, k, batch whose operands and
                 output already have GEMM layouts (no transposes): the floor
                 the transposes add to
      torch      torch.einsum on the same buffers plus the alpha/beta update
                 (its own permute copies and GEMM), full f32 (no TF32)."""
    import torch
    import hptt_b200 as h
    from hptt_b200 import workloads as w

    torch.backends.cuda.matmul.allow_tf32 = False
    cases = w.contraction_cases()
    g = torch.Generator(device="cuda").manual_seed(99)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def rnd(n, dt):
        t = _tdtype(torch, dt)
        if dt in ("c64", "c128"):
            rt = torch.float32 if dt == "c64" else torch.float64
            return torch.view_as_complex(torch.rand(n, 2, generator=g, device="cuda",
                                                    dtype=rt) * 2 - 1)
        return torch.rand(n, generator=g, device="cuda", dtype=t) * 2 - 1

    def timed(fn, reps=args.contract_reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    rows = []
    tot = {"flops": 0, "ours": 0.0, "gemm": 0.0, "torch": 0.0}
    for c in cases:
        dt = c["dtype"]
        na, nb, nc = (int(np.prod(c[k])) for k in ("size_a", "size_b", "size_c"))
        A, B, C = rnd(na, dt), rnd(nb, dt), rnd(nc, dt)
        plan = h.create_contraction(A, B, C, c["size_a"], c["labels_a"], c["size_b"],
                                    c["labels_b"], c["labels_c"], c["alpha"], c["beta"],
                                    dtype=dt)
        info = plan.info()
        ours = timed(lambda: plan.exec_on(sptr))
        info = plan.info()
        # the same GEMM with every tensor already in GEMM layout
        m, n, k, bt = info["m"], info["n"], info["k"], info["batch"]
        A2, B2, C2 = rnd(m * k * bt, dt), rnd(k * n * bt, dt), rnd(m * n * bt, dt)
        gplan = h.create_contraction(A2, B2, C2, [m, k, bt], "mkb", [k, n, bt], "knb", "mnb",
                                     c["alpha"], c["beta"], dtype=dt)
        assert gplan.info()["transposes"] == 0
        gemm = timed(lambda: gplan.exec_on(sptr))
        # torch.einsum on the same column-major buffers: reversed dims, row-major views
        sa, sb, sc = ("".join(reversed(c[k])) for k in ("labels_a", "labels_b", "labels_c"))
        Av = A.view(list(reversed(c["size_a"])))
        Bv = B.view(list(reversed(c["size_b"])))
        Cv = C.view(list(reversed(c["size_c"])))
        al, be = c["alpha"], c["beta"]

        def torch_step():
            r = torch.einsum(f"{sa},{sb}->{sc}", Av, Bv)
            if be != 0.0:
                Cv.mul_(be).add_(r, alpha=al)
            else:
                Cv.copy_(r.mul_(al) if al != 1.0 else r)
        tms = timed(torch_step)
        fl = info["flops"]
        rows.append({"dtype": dt, "spec": f"{''.join(c['labels_a'])},{''.join(c['labels_b'])}"
                                          f"->{''.join(c['labels_c'])}",
                     "size_a": c["size_a"], "size_b": c["size_b"],
                     "m": m, "n": n, "k": k, "batch": bt, "transposes": info["transposes"],
                     "transpose_bytes": info["transpose_bytes"],
                     "ms": round(ours, 4), "gemm_only_ms": round(gemm, 4),
                     "torch_einsum_ms": round(tms, 4),
                     "tflops": round(fl / ours / 1e9, 2),
                     "transpose_share": round(max(0.0, 1 - gemm / ours), 4),
                     "speedup_vs_torch": round(tms / ours, 3)})
        tot["flops"] += fl
        tot["ours"] += ours
        tot["gemm"] += gemm
        tot["torch"] += tms
        plan.destroy()
        gplan.destroy()
        del A, B, C, A2, B2, C2
    return {"workload": f"{len(cases)} seeded synthetic contractions (f32/f64, one c64, one "
                        "c128; 1-3 M/N/K labels, 0-1 batch label, random label orders; "
                        "GEMM m, n ~ 1-4 K, k ~ 0.5-2 K)",
            "api": "hptt_cuda_contract_exec_on (CUDA graph replay)",
            "total_ms": round(tot["ours"], 4), "gemm_only_ms": round(tot["gemm"], 4),
            "torch_einsum_ms": round(tot["torch"], 4),
            "tflops": round(tot["flops"] / tot["ours"] / 1e9, 2),
            "transpose_share": round(max(0.0, 1 - tot["gemm"] / tot["ours"]), 4),
            "speedup_vs_torch_einsum": round(tot["torch"] / tot["ours"], 3),
            "reps": args.contract_reps, "cases": rows}


# --------------------------------------------------------------------------
# CPU reference
# --------------------------------------------------------------------------
def _host_has_avx2():
    try:
        return "avx2" in open("/proc/cpuinfo").read()
    except Exception:
        return False


def _fill(x: np.ndarray, seed: int):
    """Cheap deterministic fill: a small random block tiled over the buffer."""
    rng = np.random.default_rng(seed)
    blk = rng.uniform(-1, 1, 1 << 16)
    flat = x.view(np.float32 if x.dtype in (np.float32, np.complex64) else np.float64)
    reps = -(-flat.size // blk.size)
    flat[:] = np.tile(blk.astype(flat.dtype), reps)[:flat.size]


class _HostBuffers:
    """One page-aligned A/B pair of the largest footprint a workload needs,
    filled once; every case runs on leading views of it (the reference's CPU
    time depends on the shape, not on the values)."""

    def __init__(self, cases):
        import oracle
        from hptt_b200.workloads import ELEM
        nbytes = max(int(np.prod(c["in_size"])) * ELEM[c["dtype"]] for c in cases)
        n = (nbytes + 15) // 16 * 2  # float64 words, a whole number of 16-byte elements
        self.a = oracle.aligned_empty(n, np.float64)
        self.b = oracle.aligned_empty(n, np.float64)
        _fill(self.a, 1)
        _fill(self.b, 2)

    def views(self, c):
        import oracle
        dt = oracle.NP_DTYPES[c["dtype"]]
        n = int(np.prod(c["in_size"]))
        return self.a.view(dt)[:n], self.b.view(dt)[:n]


def reference_time_case(c, threads, repeat=2, bufs=None):
    """Best-of-`repeat` time of one case on the reference's CPU code: its
    optimised plan where that plan is correct for the shape, else its naive
    RefTrans (labelled "naive")."""
    import oracle
    name = c["dtype"]
    a, b = (bufs or _HostBuffers([c])).views(c)
    al, be = c["alpha"], c["beta"]
    if isinstance(al, complex) or isinstance(be, complex):
        # complex scalars are not expressible through the reference API: time
        # the reference naive transpose with the real parts (same traffic)
        t = oracle.ref_naive_exec(a, b, c["in_size"], c["perm"], complex(al).real,
                                  complex(be).real, threads=threads, repeat=repeat)
        return t, "naive"
    if oracle.ref_plan_is_safe(name, c["in_size"], c["perm"], be):
        t = oracle.ref_plan_exec(a, b, c["in_size"], c["perm"], al, be, threads=threads,
                                 repeat=repeat)
        return t, "plan"
    t = oracle.ref_naive_exec(a, b, c["in_size"], c["perm"], al, be, threads=threads,
                              repeat=repeat)
    return t, "naive"


def _ref_ready():
    import oracle
    if not oracle.ref_available():
        return "oracle/_ref/libhptt_ref.so not built"
    if not _host_has_avx2():
        return "host CPU lacks AVX2 (reference AVX2 build)"
    return None


def cpu_baseline_sample(cases, budget_s=20.0, threads=None):
    from hptt_b200.workloads import algorithmic_bytes
    why = _ref_ready()
    if why:
        return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: " + why}
    threads = threads or os.cpu_count() or 1
    bufs = _HostBuffers(cases)
    t_start = time.time()
    tot_b = tot_t = 0.0
    used = {"plan": 0, "naive": 0}
    done = 0
    order = list(range(0, len(cases), 7)) + [i for i in range(len(cases)) if i % 7]
    for i in order:
        if time.time() - t_start > budget_s:
            break
        t, how = reference_time_case(cases[i], threads, bufs=bufs)
        tot_b += algorithmic_bytes(cases[i])
        tot_t += t
        used[how] += 1
        done += 1
    return {"value": round(tot_b / tot_t / 1e9, 2) if tot_t else None, "unit": "GB/s",
            "cores": threads, "kind": "reference",
            "sample": (f"{done} of {len(cases)} transposes of the same workload, best of 2 execs "
                       f"each, {threads} OpenMP threads; {used['plan']} by the reference plan, "
                       f"{used['naive']} by the reference's naive RefTrans (plan incorrect on "
                       f"those shapes or complex scalars)")}


def cpu_baseline_plain(runs=5):
    """The plain single transpose on the reference's own optimised CPU plan
    (inc/hptt/cgraph/cgraph_trans.tcc:27-48; the shape is in the subset where
    that plan is correct) at 1 OpenMP thread and at every host thread: best
    of `runs` execs, an 800 MB host buffer rewritten between execs so no run
    starts with the tensors in cache."""
    import oracle
    from hptt_b200.workloads import algorithmic_bytes, plain_single
    why = _ref_ready()
    if why:
        return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: " + why}
    c = plain_single()
    assert oracle.ref_plan_is_safe(c["dtype"], c["in_size"], c["perm"], c["beta"])
    bufs = _HostBuffers([c])
    a, b = bufs.views(c)
    trash = np.empty(100 << 20, dtype=np.float64)
    nb = algorithmic_bytes(c)
    res = {}
    for threads in (1, os.cpu_count() or 1):
        best = 1e30
        for r in range(runs):
            trash.fill(float(r))
            best = min(best, oracle.ref_plan_exec(a, b, c["in_size"], c["perm"], c["alpha"],
                                                  c["beta"], threads=threads, repeat=1))
        res[threads] = nb / best / 1e9
    allc = os.cpu_count() or 1
    return {"value": round(res[allc], 2), "unit": "GB/s", "cores": allc, "kind": "reference",
            "value_1_thread": round(res[1], 2),
            "sample": (f"the whole transpose on the reference plan, best of {runs} execs with "
                       f"an 800 MB cache rewrite between execs, at 1 and {allc} OpenMP threads")}


def run_reference(args):
    """The reference arm: the reference's own CPU code (its plan where it is
    correct for the shape, else its naive RefTrans, labelled) on every
    transpose of the workload, each step the whole workload, all host
    threads.  Steps past a time budget are not run (the line says how many
    were timed)."""
    from hptt_b200.workloads import algorithmic_bytes
    cases, desc = _workload(args.workload)
    threads = os.cpu_count() or 1
    why = _ref_ready()
    if why:
        return {"impl": "reference", "unavailable": why}
    bufs = _HostBuffers(cases)
    tot_b = tot_t = 0.0
    used = {"plan": 0, "naive": 0}
    timed = 0
    t_start = time.time()
    for s in range(args.warmup + args.steps):
        if s >= args.warmup and timed and time.time() - t_start > args.ref_budget:
            break
        step_b = step_t = 0.0
        for c in cases:
            t, how = reference_time_case(c, threads, repeat=1, bufs=bufs)
            step_b += algorithmic_bytes(c)
            step_t += t
            if s >= args.warmup:
                used[how] += 1
        if s >= args.warmup:
            tot_b += step_b
            tot_t += step_t
            timed += 1
    value = tot_b / tot_t / 1e9 if tot_t else None
    sample = (f"every step the whole workload ({len(cases)} transposes; {timed} timed steps "
              f"after {args.warmup} warm-up), {threads} OpenMP threads; per step "
              f"{used['plan'] // max(1, timed)} transposes by the reference plan and "
              f"{used['naive'] // max(1, timed)} by the reference's naive RefTrans (plan "
              f"incorrect on those shapes, or complex scalars)")
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 2) if value else None,
        "unit": "GB/s", "n_gpus": 0, "steps": timed, "warmup": args.warmup,
        "ms_per_step": round(tot_t * 1e3 / max(1, timed), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.workload == "sweep" else cases[0]["dtype"],
        "data": "synthetic", "config": {"workload": desc, "threads": threads,
                                        "transposes_per_step": len(cases)},
        "cpu_baseline": {"value": round(value, 2) if value else None, "unit": "GB/s",
                         "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": round(value, 2) if value else None, "unit": "GB/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sweep", choices=["sweep", "plain", "hard"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="seconds of reference CPU time after which no further timed step "
                         "starts (--impl reference)")
    ap.add_argument("--tune-cache", default=DEFAULT_TUNE_CACHE,
                    help="autotune cache to load before planning (tiles tuned offline on "
                         "this GPU model by `python -m hptt_b200.tune_sweep`)")
    ap.add_argument("--no-tune-cache", action="store_true",
                    help="plan with the heuristic only")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-form measurement")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--batched-only", action="store_true",
                    help="measure only the batched form (with --batch-count: profiling)")
    ap.add_argument("--served-only", action="store_true",
                    help="measure only the served form (--serve-rates, --serve-seconds)")
    ap.add_argument("--no-served", action="store_true",
                    help="skip the served-form measurement")
    ap.add_argument("--serve-rates", default="10000,30000,100000,250000,500000")
    ap.add_argument("--serve-seconds", type=float, default=2.0,
                    help="arrival window per rate (60 for the full served workload)")
    ap.add_argument("--batch-reps", type=int, default=10)
    ap.add_argument("--no-sections", action="store_true",
                    help="skip the plain single transpose and hard-layout sections")
    ap.add_argument("--no-contraction", action="store_true",
                    help="skip the tensor-contraction (transpose-GEMM-transpose) section")
    ap.add_argument("--contract-reps", type=int, default=20)
    ap.add_argument("--case", type=int, default=None,
                    help="run only transpose I of the workload (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        out = run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.barrier()
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
