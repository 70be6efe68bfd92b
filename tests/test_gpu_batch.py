"""Batched solver on the GPU: independent plates of uneven size, element
type, material and supports in one persistent launch.

Checks: every plate meets the FP64-checked error bar against its own FP64
truth; results equal single-plate solves of the same plates (block-Jacobi
PCG iterates do not depend on the partition, so iteration counts agree to
one); a batch object re-solves with new loads; per-plate and batch
statistics are filled in."""
import numpy as np
import pytest

from conftest import rel_err
from plategpu import _lib, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch():
    return workloads.batch_uneven(count=12, seed=7, min_side=8, max_side=40)


def truth(oracle, wl):
    m, mat = wl.mesh, wl.material
    ke = oracle.all_ke(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t,
                       elem_t=mat.elem_t, mode=oracle.FP64)
    x, _ = oracle.truth_solve(m.nodeCount, m.elements, m.nodesPerElement, ke, wl.cons_mask, wl.F)
    return x


def probs_of(batch):
    return [_lib.Problem(w.mesh, w.material, w.coloring, w.F, w.cons_mask) for w in batch]


@pytest.mark.parametrize("kw", [
    dict(precision=_lib.PG_PREC_MIXED, preconditioner=_lib.PG_PRECOND_TWO_LEVEL,
         smoother=_lib.PG_SMOOTHER_CHEBYSHEV),
    dict(precision=_lib.PG_PREC_FP64),
])
def test_batch_matches_truth_and_single_solves(gpu_ctx, oracle, small_batch, kw):
    opts = _lib.make_options(tolerance=1e-9, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE, **kw)
    probs = probs_of(small_batch)
    xs, infos, bi = gpu_ctx.solve_batch(probs, opts)
    assert bi.count == len(small_batch) and bi.converged == len(small_batch)
    assert bi.fallbacks >= 0 and bi.phases >= 1
    assert 0 < bi.grid <= 148 and bi.solve_ms > 0 and bi.plate_ms_p50 > 0
    assert bi.plate_ms_p50 <= bi.plate_ms_p99 <= bi.plate_ms_max <= bi.solve_ms * 1.01
    for wl, pr, x, info in zip(small_batch, probs, xs, infos):
        assert info.converged and info.status == 0
        assert rel_err(x, truth(oracle, wl)) < 1e-6
        xs1, info1 = gpu_ctx.solve(pr, opts)
        assert rel_err(x, xs1) < 1e-6
        if kw.get("preconditioner", 0) == 0 and kw.get("smoother", 0) == 0:
            assert abs(info.iterations - info1.iterations) <= 1


def test_batch_object_resolves_with_new_loads(gpu_ctx, small_batch):
    opts = _lib.make_options(tolerance=1e-9, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
                             precision=_lib.PG_PREC_MIXED, preconditioner=_lib.PG_PRECOND_TWO_LEVEL,
                             smoother=_lib.PG_SMOOTHER_CHEBYSHEV)
    probs = probs_of(small_batch)
    b = gpu_ctx.batch(probs, opts)
    x0, _i0, _b0 = b.solve(opts)
    rng = np.random.default_rng(3)
    newF = []
    for wl in small_batch:
        f = (wl.F * rng.uniform(0.5, 2.0)).astype(np.float32)
        newF.append(f)
    x1, infos, bi = b.solve(opts, F=newF)
    assert bi.converged == len(small_batch)
    for wl, pr, f, x in zip(small_batch, probs, newF, x1):
        pr2 = _lib.Problem(wl.mesh, wl.material, wl.coloring, f, wl.cons_mask)
        xs1, _ = gpu_ctx.solve(pr2, opts)
        assert rel_err(x, xs1) < 1e-6
    # a None entry keeps that plate's current load
    x2, _i, _b = b.solve(opts, F=[None] * len(small_batch))
    for a, c in zip(x1, x2):
        assert rel_err(a, c) < 1e-9
    b.close()


def test_batch_rejects_options_of_another_halo(gpu_ctx, small_batch):
    probs = probs_of(small_batch[:3])
    b = gpu_ctx.batch(probs, _lib.make_options())
    with pytest.raises(_lib.PlateGPUError, match="smoother"):
        b.solve(_lib.make_options(smoother=_lib.PG_SMOOTHER_CHEBYSHEV))
    b.close()


def test_mixed_precision_falls_back_to_fp64_when_it_stagnates(gpu_ctx, oracle, small_batch):
    """The stagnation rule (three FP64 residual replacements in a row without
    halving the residual) and the FP64 re-solve.  A replacement after every
    update (reliable_interval = 1) cannot halve the residual each time, so
    the rule fires within a few updates; with the default fallback the call
    then re-solves in FP64 to the requested accuracy."""
    wl = small_batch[1]
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    kw = dict(tolerance=1e-9, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
              precision=_lib.PG_PREC_MIXED, reliable_interval=1)
    _x, raw = gpu_ctx.solve(pr, _lib.make_options(fallback=False, **kw))
    assert not raw.converged and raw.as_dict()["stop_reason"] == "stagnated"
    assert raw.iterations < 20 and raw.fallback == 0
    x, info = gpu_ctx.solve(pr, _lib.make_options(**kw))
    assert info.converged and info.fallback == 1
    assert rel_err(x, truth(oracle, wl)) < 1e-6
    probs = probs_of(small_batch[:4])
    xs, infos, bi = gpu_ctx.solve_batch(probs, _lib.make_options(**kw))
    # plates whose residual halves at every update converge without it
    assert bi.converged == 4 and bi.fallbacks == sum(inf.fallback for inf in infos) >= 1
    for w, x, inf in zip(small_batch[:4], xs, infos):
        assert inf.converged and rel_err(x, truth(oracle, w)) < 1e-6
