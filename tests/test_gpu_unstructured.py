"""Unstructured DKT meshes (a plate with two holes, Delaunay triangles,
shuffled node numbers, per-element thickness) through the same solver:
FP64 block-Jacobi PCG against the FP64 truth and the reference-precision
oracle, the fastest variant (mixed, two-level, Chebyshev) against the truth,
every grid size agreeing, nodal moments against the oracle, and a batch of
unstructured plates.  The solves stop at a relative residual of 1e-11; the
FP64 error on this mesh is about 2.5 times the relative residual."""
import numpy as np
import pytest

from conftest import max_w, rel_err
from plategpu import _lib
import unstructured as U

pytestmark = pytest.mark.gpu


def truth(oracle, wl):
    m, mat = wl.mesh, wl.material
    ke = oracle.all_ke(m.nodes, m.elements, 3, mat.E, mat.nu, mat.t, elem_t=mat.elem_t, mode=oracle.FP64)
    x, rel = oracle.truth_solve(m.nodeCount, m.elements, 3, ke, wl.cons_mask, wl.F.astype(np.float64))
    assert rel < 1e-10
    return x


def gsolve(ctx, wl, **kw):
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    return ctx.solve(pr, _lib.make_options(**kw))


@pytest.fixture(scope="module")
def wl():
    return U.workload(h=0.12)


@pytest.fixture(scope="module")
def xt(oracle, wl):
    return truth(oracle, wl)


def test_fp64_matches_truth_and_reference(gpu_ctx, oracle, wl, xt):
    x, info = gsolve(gpu_ctx, wl, tolerance=1e-11, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE)
    assert info.converged
    assert rel_err(x, xt) < 1e-6
    m, mat = wl.mesh, wl.material
    keR = oracle.all_ke(m.nodes, m.elements, 3, mat.E, mat.nu, mat.t, elem_t=mat.elem_t, mode=oracle.REF)
    bdR = oracle.invert_block_diag(oracle.block_diag(m.nodeCount, m.elements, 3, keR, oracle.REF),
                                   wl.cons_mask, oracle.REF)
    offs, flat = wl.coloring.flat()
    xr, _it, _r, conv = oracle.solve_pcg(m.nodeCount, m.elements, 3, keR, offs, flat, wl.cons_mask, bdR,
                                         wl.F.astype(np.float64), 1e-6, 20000, oracle.REF)
    assert conv and abs(max_w(x) - max_w(xr)) / abs(max_w(xr)) < 1e-4


def test_mixed_two_level_chebyshev(gpu_ctx, wl, xt):
    x, info = gsolve(gpu_ctx, wl, tolerance=1e-11, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
                     precision=_lib.PG_PREC_MIXED, preconditioner=_lib.PG_PRECOND_TWO_LEVEL,
                     smoother=_lib.PG_SMOOTHER_CHEBYSHEV)
    assert info.converged
    assert rel_err(x, xt) < 1e-6


@pytest.mark.parametrize("ctas", [24, 64, 148])
def test_grid_sizes(gpu_ctx, wl, xt, ctas):
    x, info = gsolve(gpu_ctx, wl, tolerance=1e-11, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
                     ctas=ctas, preconditioner=_lib.PG_PRECOND_TWO_LEVEL)
    assert info.converged and info.ctas == ctas
    assert rel_err(x, xt) < 1e-6


def test_moments(gpu_ctx, oracle, wl, xt):
    m, mat = wl.mesh, wl.material
    pr = _lib.Problem(m, mat, wl.coloring, wl.F, wl.cons_mask)
    got = gpu_ctx.moments(pr, xt)
    # the reference's moments use the plate's uniform thickness
    want = oracle.moments(m.nodes, m.elements, 3, mat.E, mat.nu, mat.t, xt, oracle.FP64)
    scale = max(np.abs(w).max() for w in want)
    for g, w in zip(got, want):
        assert np.abs(g - w).max() <= 1e-12 * scale


def test_batch_of_unstructured_plates(gpu_ctx, oracle):
    wls = [U.workload(h=h, seed=s) for h, s in ((0.3, 1), (0.2, 2), (0.25, 4), (0.15, 5))]
    probs = [_lib.Problem(w.mesh, w.material, w.coloring, w.F, w.cons_mask) for w in wls]
    opts = _lib.make_options(tolerance=1e-11, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
                             precision=_lib.PG_PREC_MIXED, preconditioner=_lib.PG_PRECOND_TWO_LEVEL)
    b = gpu_ctx.batch(probs, opts)
    try:
        xs, infos, bi = b.solve(opts)
    finally:
        b.close()
    assert bi.converged == len(wls)
    for w, x in zip(wls, xs):
        assert rel_err(x, truth(oracle, w)) < 1e-6
