"""Autotuner for the batched kernel's panel width per size bucket.

The batched kernel factors each matrix with a block size taken from a table
indexed by size bucket (n <= 32, 64, 128, 256, 512, 1024).  ``autotune_batched``
times every candidate width on synthetic KKT batches of each bucket on the
current GPU and writes the fastest per bucket to ``batched_blocks.json`` next to
this file; ``load_table`` reads it back (``None`` when absent: the library's
built-in defaults apply).  A width that would not fit shared memory is
clamped by the library, so candidates that clamp to the same width are
timed once.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE_PATH = os.path.join(HERE, "batched_blocks.json")
BUCKETS = ((1, 32), (33, 64), (65, 128), (129, 256), (257, 512), (513, 1024))
CANDIDATES = (4, 8, 12, 16, 24, 32, 48, 64)


def load_table(path: str = TABLE_PATH):
    """The tuned block size per bucket, or None."""
    try:
        with open(path) as fh:
            table = json.load(fh)["table"]
    except (OSError, ValueError, KeyError):
        return None
    if len(table) != len(BUCKETS):
        return None
    return [int(v) for v in table]


def kkt_batch_device(sizes, seed: int, device, h_fraction: float = 0.75, ridge: float = 1e-2):
    """Packed KKT matrices [[H, B^T], [B, 0]] (H = G G^T / h + ridge I, G and B
    Gaussian, h = h_fraction * n) in the batched layout, plus right-hand
    sides ~ N(0, 1).  Returns (a, x) flat float64 CUDA tensors."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    sizes = [int(n) for n in sizes]
    a = torch.zeros(sum(n * n for n in sizes), dtype=torch.float64, device=device)
    off = 0
    for n in sizes:
        h = max(1, min(n, int(round(h_fraction * n))))
        m = a[off:off + n * n].view(n, n)
        gm = torch.randn(h, h, generator=g, dtype=torch.float64, device=device)
        m[:h, :h] = gm @ gm.T / h + ridge * torch.eye(h, dtype=torch.float64, device=device)
        if h < n:
            bm = torch.randn(n - h, h, generator=g, dtype=torch.float64, device=device)
            m[h:, :h] = bm
            m[:h, h:] = bm.T
        off += n * n
    x = torch.randn(sum(sizes), generator=g, dtype=torch.float64, device=device)
    return a, x


def _time_batch(bbk, sizes, block, a0, x0, reps: int) -> tuple[float, list]:
    import torch
    plan = bbk.BatchedPlan(sizes, block_sizes=[block] * len(BUCKETS))
    a = torch.empty_like(a0)
    x = torch.empty_like(x0)
    times = []
    for r in range(reps + 1):
        a.copy_(a0)
        x.copy_(x0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        bbk.batched_factor_solve(plan, a, x, mode="fp64", sync=False)
        e1.record()
        torch.cuda.synchronize()
        if r > 0:
            times.append(e0.elapsed_time(e1))
    return float(np.median(times)), [int(b) for b in plan.block_sizes]


def autotune_batched(per_bucket: int = 296, seed: int = 7, candidates=CANDIDATES, reps: int = 3,
                     write: bool = True, path: str = TABLE_PATH) -> dict:
    """Time each candidate width per bucket; returns (and optionally writes)
    {"table": [...], "ms": {bucket: {width: ms}}, "device": name}."""
    import torch

    import blockedbunchkaufmanldlt_b200 as bbk
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(seed)
    table, detail = [], {}
    for bi, (lo, hi) in enumerate(BUCKETS):
        count = per_bucket if hi <= 512 else max(148, per_bucket // 2)
        sizes = [int(v) for v in rng.integers(max(lo, 16 if hi > 16 else lo), hi + 1, size=count)]
        a0, x0 = kkt_batch_device(sizes, seed + bi, dev)
        seen, res = set(), {}
        for b in candidates:
            ms, used = _time_batch(bbk, sizes, b, a0, x0, reps)
            key = tuple(sorted(set(used)))
            if key in seen:
                continue
            seen.add(key)
            res[b] = ms
        best = min(res, key=res.get)
        table.append(int(best))
        detail[f"{lo}-{hi}"] = {str(k): round(v, 4) for k, v in res.items()}
        del a0, x0
    out = {"table": table, "ms": detail, "device": torch.cuda.get_device_name(dev),
           "candidates": list(candidates), "per_bucket": per_bucket,
           "when": time.strftime("%Y-%m-%d %H:%M:%S")}
    if write:
        with open(path, "w") as fh:
            json.dump(out, fh, indent=1)
    return out


if __name__ == "__main__":
    print(json.dumps(autotune_batched(), indent=1))
