"""Persistent PCG solve on the GPU against the oracle.

Bars: the FP64 truth x* (sparse LU + FP64 refinement of the same FP64
operator) and the reference-precision oracle (the reference CPU solver's
arithmetic, maxIterations raised so it converges).  Tolerances in each test:
relative L2 error vs x*, and |max w - max w_ref| / |max w_ref| < 1e-4 (the
reference's 0.01% rule, RULES.md:46-50).
"""
import numpy as np
import pytest

from conftest import max_w, rel_err
from plategpu import (GPUSolverOptions, PlateGPUError, _lib, coloring, mesher, problem,
                      solveGPU, workloads)
from plategpu.types import ElementColoring, PlateMaterial, PlateMesh, PlateSupport

pytestmark = pytest.mark.gpu


def oracle_setup(oracle, wl, mode):
    m, mat = wl.mesh, wl.material
    npe = m.nodesPerElement
    ke = oracle.all_ke(m.nodes, m.elements, npe, mat.E, mat.nu, mat.t, elem_t=mat.elem_t,
                       mode=mode)
    bd = oracle.invert_block_diag(oracle.block_diag(m.nodeCount, m.elements, npe, ke, mode),
                                  wl.cons_mask, mode)
    offs, flat = wl.coloring.flat()
    return ke, bd, offs, flat


def oracle_pcg(oracle, wl, tol, maxit, mode):
    ke, bd, offs, flat = oracle_setup(oracle, wl, mode)
    m = wl.mesh
    return oracle.solve_pcg(m.nodeCount, m.elements, m.nodesPerElement, ke, offs, flat,
                            wl.cons_mask, bd, wl.F.astype(np.float64), tol, maxit, mode)


def truth(oracle, wl):
    ke, _bd, _o, _f = oracle_setup(oracle, wl, oracle.FP64)
    m = wl.mesh
    x, rel = oracle.truth_solve(m.nodeCount, m.elements, m.nodesPerElement, ke, wl.cons_mask,
                                wl.F.astype(np.float64))
    assert rel < 1e-10
    return x


def gsolve(ctx, wl, **kw):
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    return ctx.solve(pr, _lib.make_options(**kw))


@pytest.fixture(scope="module")
def c1():
    return workloads.plate_q4_32()


@pytest.fixture(scope="module")
def c2():
    return workloads.plate_q4_141()


def test_q4_32_fp64(gpu_ctx, oracle, c1):
    x, info = gsolve(gpu_ctx, c1, tolerance=1e-8, max_iterations=20000,
                     stop_rule=_lib.PG_STOP_RELATIVE)
    assert info.converged and info.stop_reason == 0
    xs = truth(oracle, c1)
    assert rel_err(x, xs) < 1e-6
    assert info.true_rel_residual < 1e-7
    _xo, it_o, _r, conv = oracle_pcg(oracle, c1, 1e-8, 20000, oracle.FP64)
    assert conv and abs(info.iterations - it_o) <= 0.02 * it_o + 3
    xr, it_r, _r, conv_r = oracle_pcg(oracle, c1, 1e-6, 20000, oracle.REF)
    assert conv_r
    assert abs(max_w(x) - max_w(xr)) / abs(max_w(xr)) < 1e-4


def test_q4_141_fp64(gpu_ctx, oracle, c2):
    x, info = gsolve(gpu_ctx, c2, tolerance=7e-7, max_iterations=20000,
                     stop_rule=_lib.PG_STOP_RELATIVE)
    assert info.converged
    xs = truth(oracle, c2)
    err = rel_err(x, xs)
    assert err < 1e-6, err
    assert info.true_rel_residual < 1e-6
    xr, it_r, _r, conv_r = oracle_pcg(oracle, c2, 1e-6, 20000, oracle.REF)
    assert conv_r
    assert abs(max_w(x) - max_w(xr)) / abs(max_w(xr)) < 1e-4


@pytest.mark.parametrize("maxit", [1, 2, 5, 25])
def test_early_iterates_match_textbook_pcg(gpu_ctx, oracle, c1, maxit):
    """Chronopoulos-Gear PCG reproduces the reference's PCG iterates."""
    x, info = gsolve(gpu_ctx, c1, tolerance=0.0, max_iterations=maxit)
    xo, it_o, res_o, conv_o = oracle_pcg(oracle, c1, 0.0, maxit, oracle.FP64)
    assert info.iterations == it_o == maxit and not info.converged
    assert info.stop_reason == 1
    assert rel_err(x, xo) < 1e-10
    assert abs(info.final_residual - res_o) <= 1e-9 * res_o


def test_reference_defaults_semantics(gpu_ctx, oracle, c1):
    """Default options: tol 1e-6 on ||r|| (absolute or relative), 1000 iterations."""
    x, info = gsolve(gpu_ctx, c1)
    xo, it_o, res_o, conv_o = oracle_pcg(oracle, c1, 1e-6, 1000, oracle.FP64)
    assert bool(info.converged) == conv_o
    assert abs(info.iterations - it_o) <= 0.02 * it_o + 3


def test_zero_rhs(gpu_ctx, c1):
    wl = workloads.plate_q4_32()
    wl.F = np.zeros_like(wl.F)
    x, info = gsolve(gpu_ctx, wl)
    assert info.iterations == 0 and info.converged and info.stop_reason == 3
    assert np.all(x == 0)


def test_max_iterations_zero(gpu_ctx, c1):
    x, info = gsolve(gpu_ctx, c1, max_iterations=0)
    assert info.iterations == 0 and not info.converged
    assert abs(info.final_residual - np.linalg.norm(c1.F.astype(np.float64))) < 1e-6 * info.b_norm
    assert np.all(x == 0)


def test_breakdown_without_elements(gpu_ctx, oracle):
    """No elements: p.Ap = 0 at the first iteration -> iterations 1, not converged."""
    m = PlateMesh(nodes=np.array([0, 0, 1, 0, 1, 1, 0, 1], np.float32),
                  elements=np.zeros(0, np.uint32), boundaryNodes=np.zeros(0, np.uint32),
                  nodeCount=4, elementCount=0, nodesPerElement=4)
    F = np.zeros(12, np.float32)
    F[3] = 5.0
    pr = _lib.Problem(m, PlateMaterial(2.1e11, 0.3, 0.1), None, F, np.zeros(12, np.uint8))
    x, info = gpu_ctx.solve(pr, _lib.make_options())
    assert info.stop_reason == 2 and info.iterations == 1 and not info.converged
    assert abs(info.final_residual - 5.0) < 1e-12


def test_degenerate_triangle(gpu_ctx, oracle):
    """A zero-area triangle contributes no stiffness (element.ts:672-676)."""
    m = mesher.split_triangle_mesh(10, 10, 8, 8, jitter=0.0)
    nodes = m.nodes.copy().reshape(-1, 2)
    el = m.elements.reshape(-1, 3).copy()
    el[5] = [el[5][0], el[5][0], el[5][1]]  # repeated node: area 0
    m2 = PlateMesh(nodes=nodes.reshape(-1), elements=el.reshape(-1),
                   boundaryNodes=m.boundaryNodes, nodeCount=m.nodeCount,
                   elementCount=m.elementCount, nodesPerElement=3)
    c = coloring.computeElementColoringGreedy(m2)
    cons = problem.identifyConstrainedDOFs(m2, [PlateSupport("fixed", "all_edges")])
    F = problem.pressure_load_vector(m2, 1e3).astype(np.float32)
    problem.applyBCsToRHS(F, cons)
    wl = workloads.Workload("deg", m2, PlateMaterial(2.1e11, 0.3, 0.1), c,
                            [PlateSupport("fixed", "all_edges")], cons, F)
    x, info = gsolve(gpu_ctx, wl, tolerance=1e-10, max_iterations=5000,
                     stop_rule=_lib.PG_STOP_RELATIVE)
    assert info.converged
    assert rel_err(x, truth(oracle, wl)) < 1e-6


def test_dkt_thickness_field(gpu_ctx, oracle):
    m = mesher.split_triangle_mesh(10, 10, 40, 40, jitter=0.2, seed=9)
    rng = np.random.default_rng(9)
    et = np.clip(0.1 * (1 + 0.3 * rng.standard_normal(m.elementCount)), 0.05, 0.15)
    mat = PlateMaterial(2.1e11, 0.3, 0.1, elem_t=et.astype(np.float32))
    c = coloring.computeElementColoringGreedy(m)
    sup = [PlateSupport("fixed", "all_edges")]
    cons = problem.identifyConstrainedDOFs(m, sup)
    F = problem.pressure_load_vector(m, 3e3).astype(np.float32)
    problem.applyBCsToRHS(F, cons)
    wl = workloads.Workload("dkt40", m, mat, c, sup, cons, F)
    x, info = gsolve(gpu_ctx, wl, tolerance=1e-9, max_iterations=20000,
                     stop_rule=_lib.PG_STOP_RELATIVE)
    assert info.converged
    assert rel_err(x, truth(oracle, wl)) < 1e-6
    xr, _it, _r, conv = oracle_pcg(oracle, wl, 1e-6, 20000, oracle.REF)
    assert conv and abs(max_w(x) - max_w(xr)) / abs(max_w(xr)) < 1e-4


def test_too_few_blocks_runs_on_the_global_path(gpu_ctx, oracle, c1):
    """The whole part of a block must fit in shared memory; one block cannot
    hold 3,267 DOF, so the solve runs as flexible PCG over global memory
    (pg_info.global_path) and still meets the error bar."""
    x, info = gsolve(gpu_ctx, c1, ctas=1, tolerance=1e-9, max_iterations=20000,
                     stop_rule=_lib.PG_STOP_RELATIVE)
    assert info.global_path == 1 and info.converged
    assert rel_err(x, truth(oracle, c1)) < 1e-6
    # the smoothing-step preconditioner the faster options select on this path
    x2, info2 = gsolve(gpu_ctx, c1, ctas=1, tolerance=1e-9, max_iterations=20000,
                       stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=_lib.PG_PRECOND_TWO_LEVEL)
    assert info2.global_path == 1 and info2.converged and info2.iterations < info.iterations
    assert rel_err(x2, truth(oracle, c1)) < 1e-6


@pytest.mark.parametrize("ctas", [3, 13, 64, 148])
def test_grid_sizes_agree(gpu_ctx, c1, ctas):
    x0, i0 = gsolve(gpu_ctx, c1, tolerance=1e-8, max_iterations=5000,
                    stop_rule=_lib.PG_STOP_RELATIVE, ctas=9)
    x, info = gsolve(gpu_ctx, c1, tolerance=1e-8, max_iterations=5000,
                     stop_rule=_lib.PG_STOP_RELATIVE, ctas=ctas)
    assert info.ctas == min(ctas, c1.mesh.nodeCount)
    assert abs(info.iterations - i0.iterations) <= 3
    assert rel_err(x, x0) < 1e-8


def test_deterministic(gpu_ctx, c1):
    x1, _ = gsolve(gpu_ctx, c1, tolerance=1e-8, stop_rule=_lib.PG_STOP_RELATIVE)
    x2, _ = gsolve(gpu_ctx, c1, tolerance=1e-8, stop_rule=_lib.PG_STOP_RELATIVE)
    np.testing.assert_array_equal(x1, x2)


def test_conflicting_coloring_is_recolored(gpu_ctx, c1):
    one = ElementColoring(colors=[np.arange(c1.mesh.elementCount, dtype=np.uint32)],
                          elementColors=np.zeros(c1.mesh.elementCount, np.uint8), colorCount=1)
    wl = workloads.Workload("c1", c1.mesh, c1.material, one, c1.supports, c1.constrainedDOFs,
                            c1.F)
    x1, _ = gsolve(gpu_ctx, c1, tolerance=1e-8, stop_rule=_lib.PG_STOP_RELATIVE)
    x2, _ = gsolve(gpu_ctx, wl, tolerance=1e-8, stop_rule=_lib.PG_STOP_RELATIVE)
    assert rel_err(x2, x1) < 1e-8


def test_nonfinite_rhs_rejected(gpu_ctx, c1):
    wl = workloads.plate_q4_32()
    wl.F = wl.F.copy()
    wl.F[100] = np.nan
    with pytest.raises(PlateGPUError, match="PG_ENONFINITE"):
        gsolve(gpu_ctx, wl)


def test_wait_timeout_reports_and_context_survives(gpu_ctx, c1):
    """Block 0 waits for a value no block ever writes: the wait runs out
    after its 20 ms limit, every block leaves, the call returns
    PG_ETIMEOUT (no trap, no hang) and the context stays usable."""
    with pytest.raises(PlateGPUError, match="PG_ETIMEOUT"):
        gsolve(gpu_ctx, c1, wait_timeout_ms=20.0, ctas=16, test_stall=True)
    x, info = gsolve(gpu_ctx, c1, tolerance=1e-8, max_iterations=5000,
                     stop_rule=_lib.PG_STOP_RELATIVE)
    assert info.converged


def test_solveGPU_interface(c1):
    res = solveGPU(c1.mesh, c1.material, c1.coloring, c1.F, c1.constrainedDOFs,
                   GPUSolverOptions(tolerance=1e-8, maxIterations=5000))
    assert res.usedGPU and res.converged and res.gpuTimeMs > 0
    assert res.solution.dtype == np.float32 and res.solution.size == 3267
    with pytest.raises(PlateGPUError):
        solveGPU(c1.mesh, c1.material, c1.coloring, c1.F, c1.constrainedDOFs,
                 GPUSolverOptions(forceCPU=True))


def test_plan_cache_reused(gpu_ctx, c1):
    pr = _lib.Problem(c1.mesh, c1.material, c1.coloring, c1.F, c1.cons_mask)
    o = _lib.make_options(ctas=11)
    gpu_ctx.solve(pr, o)
    pr.set_F(c1.F * 2)
    x, info = gpu_ctx.solve(pr, o)
    assert info.plan_cached == 1


def test_plan_cache_compares_every_array(gpu_ctx, c1):
    """A plan is reused for a problem equal in every mesh, colouring,
    constraint and material array (copies in other memory included), and
    not when any one of them differs -- here the last node coordinate, the
    last colour list entry, one constraint and the thickness."""
    o = _lib.make_options(ctas=13, tolerance=1e-8, stop_rule=_lib.PG_STOP_RELATIVE)
    m, mat = c1.mesh, c1.material
    gpu_ctx.solve(_lib.Problem(m, mat, c1.coloring, c1.F, c1.cons_mask), o)
    copy = type(m)(**{**m.__dict__, "nodes": m.nodes.copy(), "elements": m.elements.copy()})
    _x, info = gpu_ctx.solve(_lib.Problem(copy, mat, c1.coloring, c1.F, c1.cons_mask.copy()), o)
    assert info.plan_cached == 1
    nodes = m.nodes.copy()
    nodes[-1] += np.float32(1e-3)
    moved = type(m)(**{**m.__dict__, "nodes": nodes})
    _x, info = gpu_ctx.solve(_lib.Problem(moved, mat, c1.coloring, c1.F, c1.cons_mask), o)
    assert info.plan_cached == 0
    cons = c1.cons_mask.copy()
    free = np.flatnonzero(cons == 0)
    cons[free[len(free) // 2]] = 1
    F = c1.F.copy()
    F[cons != 0] = 0
    _x, info = gpu_ctx.solve(_lib.Problem(m, mat, c1.coloring, F, cons), o)
    assert info.plan_cached == 0
    thin = PlateMaterial(mat.E, mat.nu, mat.t * 0.5)
    _x, info = gpu_ctx.solve(_lib.Problem(m, thin, c1.coloring, c1.F, c1.cons_mask), o)
    assert info.plan_cached == 0
    colors = [c.copy() for c in c1.coloring.colors]
    colors[-1] = colors[-1][::-1].copy()  # same colouring, other order within a colour
    col2 = ElementColoring(colors, c1.coloring.elementColors, c1.coloring.colorCount)
    _x, info = gpu_ctx.solve(_lib.Problem(m, mat, col2, c1.F, c1.cons_mask), o)
    assert info.plan_cached == 0


def test_first_solve_reports_its_set_up_phases(c1):
    """A solve in a new context times its one-time steps (partition plan,
    coarse space, eigenvalue estimate); the next solve of the same plate
    reuses them and reports zeros."""
    kw = dict(tolerance=1e-8, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
              preconditioner=_lib.PG_PRECOND_TWO_LEVEL, smoother=_lib.PG_SMOOTHER_CHEBYSHEV)
    ctx = _lib.Context(0)
    try:
        _x, first = gsolve(ctx, c1, **kw)
        assert first.converged and first.plan_cached == 0
        assert first.plan_ms > 0 and first.coarse_ms > 0 and first.eigen_ms > 0
        assert first.plan_ms + first.coarse_ms + first.eigen_ms < first.total_ms
        _x, again = gsolve(ctx, c1, **kw)
        assert again.plan_cached == 1 and again.plan_ms == 0 and again.coarse_ms == 0 and again.eigen_ms == 0
    finally:
        ctx.close()
