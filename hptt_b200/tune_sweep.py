"""Offline autotuning: tune every plan of a workload on this GPU and write the
autotune cache, so later processes pick the tuned tiles without timing
anything (plans created with tuning_timeout == 0 look the cache up).

    python -m hptt_b200.tune_sweep --out hptt_b200/tune/b200.cache \
        [--workloads sweep,plain,hard,batch] [--batch-count 4096]

Entries are keyed by (GPU name, dtype, fused rank, fused perm, size class,
whether B is read, floor(log2) of every fused extent), so one entry serves
every shape of that class.  Buffers
are allocated per case and freed before the next one.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

import hptt_b200 as h
from hptt_b200 import workloads as w


def _cases(names, batch_count):
    out = []
    for name in names:
        if name == "sweep":
            for c in w.sweep_cases():
                out.append(dict(c, alpha=1.0, beta=0.0))
                out.append(dict(c, alpha=2.3, beta=4.2))
        elif name == "plain":
            out.append(w.plain_single())
        elif name == "hard":
            out.extend(w.hard_cases())
        elif name == "batch":
            out.extend(w.batch_cases(count=batch_count))
        else:
            raise SystemExit(f"unknown workload {name}")
    return out


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--workloads", default="sweep,plain,hard")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--timeout", type=float, default=-1.0,
                    help="per-plan tuning budget in seconds (< 0: every candidate)")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    if os.path.exists(a.out):
        h.tune_cache_load(a.out)
    cases = _cases(a.workloads.split(","), a.batch_count)
    t0 = time.time()
    done = set()
    tdt = {"f32": torch.float32, "f64": torch.float64, "c64": torch.complex64,
           "c128": torch.complex128}
    for i, c in enumerate(cases):
        n = int(np.prod(c["in_size"]))
        al, be = c["alpha"], c["beta"]
        key = (c["dtype"], tuple(c["in_size"]), tuple(c["perm"]), be != 0)
        if key in done:
            continue
        done.add(key)
        x = torch.zeros(n, dtype=tdt[c["dtype"]], device="cuda")
        y = torch.zeros_like(x)
        p = h.create_plan(x, y, c["in_size"], c["perm"], al, be, 0, a.timeout,
                          dtype=c["dtype"])
        if p is None:
            print(f"[{i}] {c['dtype']} {c['in_size']} {c['perm']}: plan refused", flush=True)
        del p, x, y
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    h.tune_cache_save(a.out)
    print(f"tuned {len(done)} plans in {time.time() - t0:.1f} s; "
          f"{h.tune_cache_size()} cache entries -> {a.out}", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
