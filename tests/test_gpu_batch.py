"""Batched solver on the GPU: independent plates of uneven size, element
type, material and supports in one persistent launch.

Checks: every plate meets the FP64-checked error bar against its own FP64
truth; results equal single-plate solves of the same plates (block-Jacobi
PCG iterates do not depend on the partition in exact arithmetic; the
partition and the block's thread count set the summation order of the
dot products, and over a thousand FP64 iterations that rounding moves the
stop by up to about 1%, so the counts agree to 2%); a batch object
re-solves with new loads; per-plate and batch statistics are filled in."""
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
    assert bi.graph == 1  # the phase launches ran as one captured CUDA graph
    assert 0 < bi.grid <= 148 and bi.solve_ms > 0 and bi.plate_ms_p50 > 0
    assert bi.plate_ms_p50 <= bi.plate_ms_p99 <= bi.plate_ms_max <= bi.solve_ms * 1.01
    for wl, pr, x, info in zip(small_batch, probs, xs, infos):
        assert info.converged and info.status == 0
        assert rel_err(x, truth(oracle, wl)) < 1e-6
        xs1, info1 = gpu_ctx.solve(pr, opts)
        assert rel_err(x, xs1) < 1e-6
        if kw.get("preconditioner", 0) == 0 and kw.get("smoother", 0) == 0:
            assert abs(info.iterations - info1.iterations) <= max(1, 0.02 * info1.iterations)


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
    then finishes in FP64 to the requested accuracy."""
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


def oracle_true_rel(oracle, wl, x):
    """||F - K x|| / ||F|| with the oracle's FP64 operator."""
    m, mat = wl.mesh, wl.material
    ke = oracle.all_ke(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t,
                       elem_t=mat.elem_t, mode=oracle.FP64)
    offs, flat = wl.coloring.flat()
    kx = oracle.apply_k(m.nodeCount, m.elements, m.nodesPerElement, ke, offs, flat, wl.cons_mask,
                        np.asarray(x, np.float64), oracle.FP64)
    F = wl.F.astype(np.float64)
    F[wl.cons_mask != 0] = 0.0
    return float(np.linalg.norm(F - kx) / np.linalg.norm(F))


def test_fp64_correction_starts_from_the_mixed_solution(gpu_ctx, oracle, small_batch):
    """After a stagnated mixed solve the FP64 stage solves the correction
    K d = F - K x_m from the stagnated x_m: fewer iterations than an FP64
    solve from zero to the same stop, and the reported true residual is that
    of the returned x (checked with the oracle's FP64 operator).  A relative
    residual of 1e-13 is out of FP32's reach, so the mixed stage stagnates."""
    wl = workloads.plate_q4_32()
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    kw = dict(tolerance=1e-13, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE)
    x, info = gpu_ctx.solve(pr, _lib.make_options(precision=_lib.PG_PREC_MIXED, **kw))
    _x64, cold = gpu_ctx.solve(pr, _lib.make_options(precision=_lib.PG_PREC_FP64, **kw))
    assert info.fallback == 1 and info.converged and cold.converged
    assert info.iterations < 0.8 * cold.iterations
    # the true residual of the returned x; at this depth both it and the
    # oracle's value are FP64 rounding of F - K x (different summation
    # orders), so they agree to a factor, not to digits
    rel = oracle_true_rel(oracle, wl, x)
    assert 0.5 * rel <= info.true_rel_residual <= 2.0 * rel
    assert rel < 1e-11
    assert rel_err(x, truth(oracle, wl)) < 1e-6
    # the batch path: the same plate among others
    probs = probs_of(small_batch[:3]) + [pr]
    xs, infos, bi = gpu_ctx.solve_batch(probs, _lib.make_options(precision=_lib.PG_PREC_MIXED, **kw))
    assert infos[3].fallback == 1 and infos[3].converged
    assert infos[3].iterations < 0.8 * cold.iterations
    rel_b = oracle_true_rel(oracle, wl, xs[3])
    assert 0.5 * rel_b <= infos[3].true_rel_residual <= 2.0 * rel_b
    for w, xb in zip(small_batch[:3] + [wl], xs):
        assert rel_err(xb, truth(oracle, w)) < 1e-6


def test_plate_larger_than_the_first_capacity_guess_gets_the_whole_device(gpu_ctx, small_batch):
    """A 59,536-node DKT plate needs more than 400 nodes per block on 148
    blocks, above the batch's first FP64 capacity guess: it gets a team of the
    whole device with the layout a one-plate solve uses, and gives the
    one-plate solve's result (same partition, same iterates)."""
    from plategpu import coloring, mesher, problem
    from plategpu.types import PlateMaterial, PlateSupport

    m = mesher.split_triangle_mesh(10, 10, 243, 243, jitter=0.2, seed=4)
    sup = [PlateSupport("fixed", "all_edges")]
    cons = problem.identifyConstrainedDOFs(m, sup)
    F = problem.pressure_load_vector(m, 2e3).astype(np.float32)
    problem.applyBCsToRHS(F, cons)
    big = workloads.Workload("dkt243", m, PlateMaterial(2.1e11, 0.3, 0.12),
                             coloring.computeElementColoringGreedy(m), sup, cons, F)
    assert m.nodeCount > 148 * 400
    kw = dict(tolerance=1e-9, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
              precision=_lib.PG_PREC_FP64, preconditioner=_lib.PG_PRECOND_TWO_LEVEL)
    probs = probs_of([small_batch[0], small_batch[2]]) + probs_of([big])
    xs, infos, bi = gpu_ctx.solve_batch(probs, _lib.make_options(**kw))
    assert infos[2].converged and infos[2].ctas == 148
    x1, one = gpu_ctx.solve(probs[2], _lib.make_options(ctas=148, **kw))
    assert abs(infos[2].iterations - one.iterations) <= 1
    assert rel_err(xs[2], x1) < 1e-9


def test_plate_too_large_for_the_smoother_halo_runs_with_block_jacobi(gpu_ctx, small_batch):
    """With the Chebyshev smoother a 66,049-node DKT plate's 2-ring layout
    does not fit in FP64 even on the whole device: that plate runs with a
    1-ring halo and block-Jacobi smoothing (lambda_max reported 0) and gives
    the one-plate result of that method, while the other plates keep the
    smoother."""
    from plategpu import coloring, mesher, problem
    from plategpu.types import PlateMaterial, PlateSupport

    m = mesher.split_triangle_mesh(10, 10, 256, 256, jitter=0.2, seed=8)
    sup = [PlateSupport("fixed", "all_edges")]
    cons = problem.identifyConstrainedDOFs(m, sup)
    F = problem.pressure_load_vector(m, 2e3).astype(np.float32)
    problem.applyBCsToRHS(F, cons)
    big = workloads.Workload("dkt256", m, PlateMaterial(2.1e11, 0.3, 0.1),
                             coloring.computeElementColoringGreedy(m), sup, cons, F)
    kw = dict(tolerance=1e-9, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
              precision=_lib.PG_PREC_FP64, preconditioner=_lib.PG_PRECOND_TWO_LEVEL)
    probs = probs_of([small_batch[0], small_batch[2]]) + probs_of([big])
    xs, infos, bi = gpu_ctx.solve_batch(probs, _lib.make_options(smoother=_lib.PG_SMOOTHER_CHEBYSHEV, **kw))
    assert bi.converged == 3
    assert infos[0].smoother_lambda_max > 0 and infos[1].smoother_lambda_max > 0
    assert infos[2].smoother_lambda_max == 0 and infos[2].ctas == 148
    x1, one = gpu_ctx.solve(probs[2], _lib.make_options(ctas=148, **kw))
    assert abs(infos[2].iterations - one.iterations) <= 1
    assert rel_err(xs[2], x1) < 1e-9


def test_autotuner_times_candidates_and_the_schedule_follows(gpu_ctx, small_batch, tmp_path):
    """The autotuner times the batch at each part-size target on the GPU and
    caches the fastest; a larger target gives a plate fewer blocks."""
    import torch

    from plategpu import autotune

    probs = probs_of(small_batch)
    opts = _lib.make_options(tolerance=1e-9, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
                             precision=_lib.PG_PREC_FP64, preconditioner=_lib.PG_PRECOND_TWO_LEVEL)
    path = str(tmp_path / "tune.json")
    name = torch.cuda.get_device_name(0)
    best, rec = autotune.tune_batch(gpu_ctx, probs, opts, name, candidates=(64, 400), cache_path=path)
    assert best in (64, 400) and not rec["cached"] and all(v > 0 for v in rec["times_ms"].values())
    assert autotune.tune_batch(gpu_ctx, probs, opts, name, candidates=(64, 400), cache_path=path)[1]["cached"]
    few = gpu_ctx.solve_batch(probs, _lib.make_options(**{**dict(tolerance=1e-9, max_iterations=20000,
                                                                stop_rule=_lib.PG_STOP_RELATIVE),
                                                             "batch_part_nodes": 4000}))
    many = gpu_ctx.solve_batch(probs, _lib.make_options(tolerance=1e-9, max_iterations=20000,
                                                        stop_rule=_lib.PG_STOP_RELATIVE, batch_part_nodes=16))
    assert sum(i.ctas for i in few[1]) < sum(i.ctas for i in many[1])
    assert few[2].converged == many[2].converged == len(small_batch)
