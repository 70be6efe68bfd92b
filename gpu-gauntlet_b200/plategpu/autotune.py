"""Autotuner of the batched solver's launch shape.

A batch of plates (pg_batch_create) gives every plate a team of thread
blocks: at least as many as its parts need to fit in shared memory, and
otherwise about `batch_part_nodes` nodes per block (fewer blocks per plate
cost less block time, more blocks cut a plate's latency).  The best target
depends on the GPU and on the batch's size mix, so tune_batch times the
batch at each candidate target and keeps the fastest, caching the result
in a JSON file keyed by the GPU's name and a signature of the batch (plate
sizes, element types and the method's options).
"""
from __future__ import annotations

import hashlib
import json
import os
import time

from . import _lib

CANDIDATES = (250, 320, 400, 500, 640)


def default_cache_path():
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "plategpu", "batch_autotune.json")


def batch_signature(probs, opts) -> str:
    """Hash of what the launch shape depends on: each plate's node and
    element counts and element type, and the method's options."""
    h = hashlib.sha256()
    for p in probs:
        s = p.struct
        h.update(f"{s.node_count},{s.element_count},{s.nodes_per_element};".encode())
    h.update(f"{opts.precision},{opts.preconditioner},{opts.smoother}".encode())
    return h.hexdigest()[:16]


def load_cache(path):
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(path, cache):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def choose(times: dict) -> int:
    """The fastest candidate; ties go to the smaller target."""
    return min(times, key=lambda k: (times[k], int(k)))


def tune_batch(ctx, probs, opts, gpu_name, candidates=CANDIDATES, repeats=2, cache_path=None,
               time_fn=None):
    """Best batch_part_nodes for this batch and method on this GPU: from the
    cache when present, else timed (median device time of `repeats` solves
    after one warm-up solve at each candidate) and cached.  Returns (best,
    record) with record = {"times_ms": {candidate: ms}, "cached": bool, ...}.
    time_fn(part_nodes) -> ms replaces the GPU timing (tests)."""
    path = cache_path or default_cache_path()
    cache = load_cache(path)
    sig = batch_signature(probs, opts)
    rec = cache.get(gpu_name, {}).get(sig)
    if rec is not None and "best" in rec:
        out = dict(rec)
        out["cached"] = True
        return int(rec["best"]), out

    def gpu_time(part_nodes):
        o = _lib.make_options()
        import ctypes
        ctypes.memmove(ctypes.byref(o), ctypes.byref(opts), ctypes.sizeof(o))
        o.batch_part_nodes = int(part_nodes)
        b = ctx.batch(probs, o)
        try:
            b.solve(o, want_x=False)
            ms = sorted(b.solve(o, want_x=False)[2].solve_ms for _ in range(max(1, repeats)))
        finally:
            b.close()
        return ms[len(ms) // 2]

    t0 = time.time()
    fn = time_fn or gpu_time
    times = {str(int(c)): float(fn(int(c))) for c in candidates}
    best = int(choose(times))
    rec = {"best": best, "times_ms": times, "plates": len(probs), "tuned_s": time.time() - t0,
           "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
    cache.setdefault(gpu_name, {})[sig] = rec
    save_cache(path, cache)
    out = dict(rec)
    out["cached"] = False
    return best, out
