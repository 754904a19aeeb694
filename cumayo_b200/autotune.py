"""Autotuners: the persistent work queue's launch shapes and the shared-key path's block shapes.

tune_queue: for a given queue (operands already set) it times candidate launch shapes on the
actual GPU with CUDA events — the resident CTAs per SM of each (set, op) bucket's kernel and the
order in which the bucket kernels are launched (the first one launched takes the SMs first, the
later ones fill in as its CTAs finish) — and keeps the fastest.

tune_shared: for one set's sign_shared + verify_shared on a given batch it times the block shapes
the library can run — threads per CTA of the thread-per-instance hash kernels (32..256) and
signatures per sign-tail CTA (1, or 2 or 4 with the instances' elimination columns interleaved) and
CTAs per key-product tile (1, or a CTA pair sharing each tile's key rows) — and sets the fastest
(mayo_b200_shared_set_shape).

Results are cached per (GPU name, SMs, workload) in a JSON file (MAYO_B200_TUNE_CACHE, default
~/.cache/mayo_b200/autotune.json) so later runs skip the search.
"""
from __future__ import annotations

import json
import os

import numpy as np

from . import queue as Q

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
    """Item counts per (op, set) field value: the workload's mix and size."""
    counts = np.bincount((np.asarray(items, dtype=np.uint32) >> 28).astype(np.int64), minlength=16)
    return "q:" + ",".join(str(int(c)) for c in counts)


def cache_key(gpu_name: str, sms: int, per_max: dict, items: np.ndarray) -> str:
    """Cache key: the GPU, the SMs used, every bucket's resident CTAs per SM (the kernels' register
    and shared-memory budgets: a library built with other budgets must not replay shapes tuned
    for another one) and the workload signature."""
    occ = ",".join(f"{s}/{op}={per_max[(s, op)]}" for (s, op) in sorted(per_max))
    return f"{gpu_name}|sms={sms}|occ={occ}|{signature(items)}"


def clamp_shape(ctas_per_sm: dict, per_max: dict) -> dict:
    """A shape's CTAs per SM, each within 1 .. the bucket's residency."""
    return {b: max(1, min(int(c), int(per_max.get(b, c)))) for b, c in ctas_per_sm.items()}


def _time(q: "Q.Queue", repeats: int) -> float:
    import torch
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
    return min(ms)


def tune_queue(q: "Q.Queue", items: np.ndarray, repeats: int = 2, use_cache: bool = True) -> dict:
    """Pick the launch shape (CTAs per SM per (set, op) bucket, the order of the bucket kernels)
    for `q` and `items`; leaves q loaded with `items` and the chosen shape."""
    import torch
    dev = torch.cuda.current_device()
    name = torch.cuda.get_device_name(dev)
    per_max = {b: Q.ctas_per_sm(*b) for b in Q.BUCKETS}
    key = cache_key(name, q.shape.sms, per_max, items)
    cache = _load() if use_cache else {}
    q.load(items)
    if key in cache:
        best = cache[key]
    else:
        orders = {"longest_first": Q.DEFAULT_ORDER, "shortest_first": Q.DEFAULT_ORDER[::-1],
                  "by_set": list(Q.BUCKETS)}
        trials, seen = [], set()
        for oname, order in orders.items():
            for occ in (0, 1):
                cps = {b: max(1, per_max[b] - occ) for b in per_max}
                if (oname, tuple(cps.values())) in seen:
                    continue
                seen.add((oname, tuple(cps.values())))
                q.shape = Q.Shape(sms=q.shape.sms, ctas_per_sm=cps, launch_order=order)
                trials.append({"ctas_per_sm": {f"{s}/{op}": c for (s, op), c in cps.items()},
                               "launch_order": oname, "ms": _time(q, repeats)})
        best = dict(min(trials, key=lambda t: t["ms"]), trials=trials)
        best["order_buckets"] = [list(b) for b in orders[best["launch_order"]]]
        cache[key] = best
        if use_cache:
            _store(cache)
    cps = {tuple(int(x) for x in k.split("/")): c for k, c in best["ctas_per_sm"].items()}
    q.shape = Q.Shape(sms=q.shape.sms, ctas_per_sm=clamp_shape(cps, per_max),
                      launch_order=[tuple(b) for b in best["order_buckets"]])
    return best


SHARED_CANDIDATES = [(h, g, p) for p in (1, 2) for g in (1, 2, 4) for h in (32, 64, 128, 256)]


def _lib_id() -> str:
    """Digest of the library file: shapes tuned for one build are not replayed on another."""
    import hashlib
    from .api import LIB_PATH
    try:
        with open(LIB_PATH, "rb") as f:
            return hashlib.sha1(f.read()).hexdigest()[:12]
    except OSError:
        return "none"


def tune_shared(m, run, batch: int, repeats: int = 3, flush=None, use_cache: bool = True) -> dict:
    """Pick the shared-key block shape of m's set for `run()` (a callable that issues the
    sign_shared / verify_shared work being tuned, on the current stream) at `batch` instances.
    `flush()`, when given, runs before every timed call (an L2 flush).  Sets the winner."""
    import torch
    dev = torch.cuda.current_device()
    props = torch.cuda.get_device_properties(dev)
    key = f"{props.name}|sms={props.multi_processor_count}|lib={_lib_id()}|shared:set={m.set}|batch={batch}"
    cache = _load() if use_cache else {}
    if key in cache:
        best = cache[key]
    else:
        trials = []
        for h, g, p in SHARED_CANDIDATES:
            try:
                m.set_shared_shape(h, g, p)
            except Exception:  # a shape this set's kernels cannot take (shared memory)
                continue
            run()
            torch.cuda.synchronize()
            ms = []
            for _ in range(repeats):
                if flush is not None:
                    flush()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                run()
                b.record()
                torch.cuda.synchronize()
                ms.append(a.elapsed_time(b))
            trials.append({"hash_threads": h, "tail_instances": g, "product_ctas": p, "ms": min(ms)})
        best = dict(min(trials, key=lambda t: t["ms"]), trials=trials)
        cache[key] = best
        if use_cache:
            _store(cache)
    m.set_shared_shape(best["hash_threads"], best["tail_instances"], best.get("product_ctas", 1))
    return best
