"""The batch autotuner's host logic (no GPU): the fastest candidate wins,
results are cached per GPU name and batch signature, and a cached result
is returned without timing again."""
import os

from plategpu import _lib, autotune, workloads


def probs_of(ws):
    return [_lib.Problem(w.mesh, w.material, w.coloring, w.F, w.cons_mask) for w in ws]


def test_fastest_candidate_is_chosen_and_cached(tmp_path):
    ws = workloads.batch_uneven(count=4, seed=2, min_side=8, max_side=16)
    probs = probs_of(ws)
    opts = _lib.make_options(precision=_lib.PG_PREC_FP64)
    path = os.path.join(tmp_path, "tune.json")
    calls = []

    def fake(part_nodes):
        calls.append(part_nodes)
        return {250: 5.0, 400: 3.0, 640: 3.0}[part_nodes]

    best, rec = autotune.tune_batch(None, probs, opts, "GPU A", candidates=(250, 400, 640), cache_path=path,
                                    time_fn=fake)
    assert best == 400 and not rec["cached"] and calls == [250, 400, 640]
    best2, rec2 = autotune.tune_batch(None, probs, opts, "GPU A", candidates=(250, 400, 640), cache_path=path,
                                      time_fn=fake)
    assert best2 == 400 and rec2["cached"] and len(calls) == 3
    # another GPU, or another method, is tuned again
    autotune.tune_batch(None, probs, opts, "GPU B", candidates=(250,), cache_path=path, time_fn=fake)
    o2 = _lib.make_options(precision=_lib.PG_PREC_MIXED)
    autotune.tune_batch(None, probs, o2, "GPU A", candidates=(640,), cache_path=path, time_fn=fake)
    assert len(calls) == 5
    cache = autotune.load_cache(path)
    assert set(cache) == {"GPU A", "GPU B"} and len(cache["GPU A"]) == 2


def test_signature_depends_on_sizes_and_method():
    ws = workloads.batch_uneven(count=3, seed=2, min_side=8, max_side=16)
    a = autotune.batch_signature(probs_of(ws), _lib.make_options())
    b = autotune.batch_signature(probs_of(ws[:2]), _lib.make_options())
    c = autotune.batch_signature(probs_of(ws), _lib.make_options(preconditioner=_lib.PG_PRECOND_TWO_LEVEL))
    assert len({a, b, c}) == 3


def test_unreadable_cache_is_ignored(tmp_path):
    path = os.path.join(tmp_path, "bad.json")
    open(path, "w").write("{not json")
    assert autotune.load_cache(path) == {}
