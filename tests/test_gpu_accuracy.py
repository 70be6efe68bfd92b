"""Accuracy bars beyond one load and at full size.

- The fastest single-plate method (mixed precision, two-level
  preconditioner, Chebyshev smoother) at the stop the benchmark uses for it
  (||r||/||b|| < 3e-6) reaches FP64 relative L2 error <= 1e-6 on the
  plate_q4_141 load and on 8 seeded random-field loads (Gaussian random
  field pressure + 0-16 point loads), not only on the one load it is timed
  on.
- plate_dkt_200 at its own size (121,203 DOF, jittered DKT, random-field
  thickness) in FP64 and in mixed precision: FP64 error <= 1e-6 and max w
  within 1e-4 of the reference-precision CPU solve (the reference's 0.01%
  rule, RULES.md:46-50).
- A batch with a DKT plate of about 30k nodes with the Chebyshev smoother in
  FP64, the size range where the first team guess is 128 blocks: it
  converges and matches the one-plate solve.
"""
import numpy as np
import pytest

from conftest import max_w, rel_err
from plategpu import _lib, workloads

pytestmark = pytest.mark.gpu


def fp64_truth_factor(oracle, wl):
    m, mat = wl.mesh, wl.material
    ke = oracle.all_ke(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t,
                       elem_t=mat.elem_t, mode=oracle.FP64)
    return oracle.truth_factor(m.nodeCount, m.elements, m.nodesPerElement, ke, wl.cons_mask)


def test_fastest_method_meets_1e6_on_eight_loads(gpu_ctx, oracle):
    wl = workloads.plate_q4_141()
    solve = fp64_truth_factor(oracle, wl)
    loads = [wl.F] + list(workloads.random_field_loads(wl, 7, seed=91))
    opts = _lib.make_options(tolerance=3e-6, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
                             precision=_lib.PG_PREC_MIXED,
                             preconditioner=_lib.PG_PRECOND_TWO_LEVEL,
                             smoother=_lib.PG_SMOOTHER_CHEBYSHEV, reliable_delta=0.01)
    errs = []
    for F in loads:
        pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, F, wl.cons_mask)
        x, info = gpu_ctx.solve(pr, opts)
        assert info.converged
        xt, rel = solve(F)
        assert rel < 1e-10
        errs.append(rel_err(x, xt))
    assert len(errs) == 8
    assert max(errs) <= 1e-6, errs


@pytest.fixture(scope="module")
def c3():
    return workloads.plate_dkt_200()


@pytest.mark.parametrize("precision", [_lib.PG_PREC_FP64, _lib.PG_PREC_MIXED])
def test_plate_dkt_200_full_size(gpu_ctx, oracle, c3, precision):
    wl = c3
    assert wl.n_dof == 121_203 and wl.mesh.elementCount == 80_000
    assert wl.material.elem_t is not None
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    x, info = gpu_ctx.solve(pr, _lib.make_options(tolerance=1e-7, max_iterations=20000,
                                                  stop_rule=_lib.PG_STOP_RELATIVE,
                                                  precision=precision))
    assert info.converged
    xt, rel = fp64_truth_factor(oracle, wl)(wl.F)
    assert rel < 1e-10
    assert rel_err(x, xt) <= 1e-6
    # the reference-precision CPU solve (maxIterations raised so it converges)
    m, mat = wl.mesh, wl.material
    ke = oracle.all_ke(m.nodes, m.elements, 3, mat.E, mat.nu, mat.t, elem_t=mat.elem_t,
                       mode=oracle.REF)
    bd = oracle.invert_block_diag(oracle.block_diag(m.nodeCount, m.elements, 3, ke, oracle.REF),
                                  wl.cons_mask, oracle.REF)
    offs, flat = wl.coloring.flat()
    xr, _it, _res, conv = oracle.solve_pcg(m.nodeCount, m.elements, 3, ke, offs, flat, wl.cons_mask,
                                           bd, wl.F.astype(np.float64), 1e-6, 20000, oracle.REF)
    assert conv
    assert abs(max_w(x) - max_w(xr)) / abs(max_w(xr)) < 1e-4


def test_batch_dkt_plate_near_the_128_block_team(gpu_ctx, oracle):
    from plategpu import coloring, mesher, problem
    from plategpu.types import PlateMaterial, PlateSupport

    m = mesher.split_triangle_mesh(10, 10, 172, 172, jitter=0.2, seed=6)
    assert 27_700 < m.nodeCount <= 32_000
    sup = [PlateSupport("fixed", "all_edges")]
    cons = problem.identifyConstrainedDOFs(m, sup)
    F = problem.pressure_load_vector(m, 2e3).astype(np.float32)
    problem.applyBCsToRHS(F, cons)
    big = workloads.Workload("dkt172", m, PlateMaterial(2.1e11, 0.3, 0.1),
                             coloring.computeElementColoringGreedy(m), sup, cons, F)
    small = workloads.batch_uneven(count=3, seed=7, min_side=8, max_side=24)
    probs = [_lib.Problem(w.mesh, w.material, w.coloring, w.F, w.cons_mask) for w in small + [big]]
    kw = dict(tolerance=1e-9, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
              precision=_lib.PG_PREC_FP64, preconditioner=_lib.PG_PRECOND_TWO_LEVEL,
              smoother=_lib.PG_SMOOTHER_CHEBYSHEV)
    xs, infos, bi = gpu_ctx.solve_batch(probs, _lib.make_options(**kw))
    assert bi.converged == 4
    xt, _ = fp64_truth_factor(oracle, big)(big.F)
    assert rel_err(xs[3], xt) < 1e-6
    x1, one = gpu_ctx.solve(probs[3], _lib.make_options(ctas=infos[3].ctas, **kw))
    assert rel_err(xs[3], x1) < 1e-7
