"""Autotuner for the persistent work queue.

For a given queue (operands already set, items loaded) it times candidate launch shapes on the
actual GPU with CUDA events — the number of resident CTAs (one or more per SM) and the item order
(as submitted, or the most expensive items first so the last CTAs do not finish a long keypair
alone) — and keeps the fastest.  Results are cached per (GPU name, workload signature) in a JSON
file (MAYO_B200_TUNE_CACHE, default ~/.cache/mayo_b200/autotune.json) so later runs skip the
search.
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import queue as Q

# Relative cost of one item per (set, op): GF(16) MACs plus 300 ops per AES block (keypair).
_PARAMS = {1: (86, 78, 8, 10, 144495), 2: (81, 64, 17, 4, 101376), 3: (118, 108, 10, 11, 376164),
           5: (154, 142, 12, 12, 841847)}


def item_cost(op: int, set_id: int) -> float:
    n, m, o, k, p = _PARAMS[set_id]
    v = n - o
    e1, e2, e3 = v * (v + 1) // 2, v * o, o * (o + 1) // 2
    if op == Q.OP_KEYPAIR:
        return o * m * (e1 + e2) + m * o * o * v + 300.0 * p / 16
    if op == Q.OP_SIGN:
        return k * m * e1 + m * k * k * v + k * m * v * o + m * m * (k * o + 1)
    return k * m * (e1 + e2 + e3) + m * k * k * n


def heavy_first(items: np.ndarray) -> np.ndarray:
    inv = {v: k for k, v in Q.SET_INDEX.items()}
    cost = np.array([item_cost(int(x) >> 30, inv[(int(x) >> 28) & 3]) for x in items])
    return items[np.argsort(-cost, kind="stable")]


def _cache_path() -> str:
    return os.environ.get("MAYO_B200_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "mayo_b200",
                                                                  "autotune.json"))


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(d: dict) -> None:
    p = _cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        with open(p, "w") as f:
            json.dump(d, f, indent=1)
    except OSError:
        pass


def signature(items: np.ndarray) -> str:
    counts = np.bincount((items >> 28).astype(np.int64), minlength=16)
    return "q:" + ",".join(str(int(c)) for c in counts)


def tune_queue(q: "Q.Queue", items: np.ndarray, repeats: int = 2, use_cache: bool = True) -> dict:
    """Pick (ctas, order) for `q` and `items`; leaves q loaded with the chosen order and shape."""
    import torch
    L = Q._bind()
    dev = torch.cuda.current_device()
    name = torch.cuda.get_device_name(dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    per_sm = max(1, L.mayo_b200_queue_ctas_per_sm())
    key = f"{name}|{signature(items)}"
    cache = _load() if use_cache else {}
    if key in cache:
        best = cache[key]
    else:
        trials = []
        for ctas in sorted({sms * c for c in range(1, per_sm + 1)}):
            if ctas > q.ctas:
                continue  # the queue memory was sized for q.ctas CTAs
            for order in ("submitted", "heavy_first"):
                arr = heavy_first(items) if order == "heavy_first" else items
                q.load(arr)
                saved = q.ctas
                q.ctas = ctas
                q.run()
                torch.cuda.synchronize()
                ms = []
                for _ in range(repeats):
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record()
                    q.run()
                    b.record()
                    torch.cuda.synchronize()
                    ms.append(a.elapsed_time(b))
                q.ctas = saved
                trials.append({"ctas": ctas, "order": order, "ms": min(ms)})
        best = min(trials, key=lambda t: t["ms"])
        best = {"ctas": best["ctas"], "order": best["order"], "ms": best["ms"], "trials": trials}
        cache[key] = best
        if use_cache:
            _store(cache)
    q.ctas = best["ctas"]
    q.load(heavy_first(items) if best["order"] == "heavy_first" else items)
    return best
