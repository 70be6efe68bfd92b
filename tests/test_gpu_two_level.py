"""Two-level preconditioner (block Jacobi + Galerkin coarse correction on
one aggregate per thread block) on the GPU.

Checks: FP64-checked error <= 1e-6 against the FP64 truth and the
reference's 0.01% max-w rule against the reference-precision CPU solve; the
iteration count matches a numpy model of the same preconditioner (the
persistent kernel's Chronopoulos-Gear recurrence and textbook PCG give the
same iterates in exact arithmetic); and the two-level method needs far
fewer iterations than block Jacobi.
"""
import numpy as np
import pytest

from conftest import max_w, rel_err
from plategpu import _lib, coloring, mesher, problem, workloads
from plategpu.types import PlateMaterial, PlateSupport
from two_level_ref import coarse_basis, strip_partition, two_level_pcg

pytestmark = pytest.mark.gpu

TL = _lib.PG_PRECOND_TWO_LEVEL


def fp64_operator(oracle, wl):
    m, mat = wl.mesh, wl.material
    npe = m.nodesPerElement
    ke = oracle.all_ke(m.nodes, m.elements, npe, mat.E, mat.nu, mat.t, elem_t=mat.elem_t,
                       mode=oracle.FP64)
    A = oracle.assemble(m.nodeCount, m.elements, npe, ke, wl.cons_mask)
    bd = oracle.invert_block_diag(oracle.block_diag(m.nodeCount, m.elements, npe, ke,
                                                    oracle.FP64), wl.cons_mask, oracle.FP64)
    b = wl.F.astype(np.float64)
    b[wl.cons_mask != 0] = 0.0
    return ke, A, bd, b


def gsolve(ctx, wl, **kw):
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    return ctx.solve(pr, _lib.make_options(**kw))


@pytest.fixture(scope="module")
def c2():
    return workloads.plate_q4_141()


@pytest.mark.parametrize("precision", [_lib.PG_PREC_FP64, _lib.PG_PREC_MIXED])
def test_two_level_q4_141(gpu_ctx, oracle, c2, precision):
    ke, A, bd, b = fp64_operator(oracle, c2)
    import scipy.sparse.linalg as spla
    xs = spla.spsolve(A.tocsc(), b)
    x, info = gsolve(gpu_ctx, c2, tolerance=5e-6, max_iterations=20000, precision=precision,
                     stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=TL)
    assert info.converged and info.coarse_dim == 3 * info.ctas
    assert rel_err(x, xs) < 1e-6
    assert info.iterations < 400  # block Jacobi needs ~1450 at this tolerance
    G = info.ctas
    part = strip_partition(c2.mesh.nodes.reshape(-1, 2).astype(np.float64), G)
    P = coarse_basis(c2.mesh.nodes.reshape(-1, 2).astype(np.float64), c2.cons_mask, part, G)
    _xm, it_m = two_level_pcg(A, b, bd, P, 5e-6)
    assert abs(info.iterations - it_m) <= 0.03 * it_m + 2
    offs, flat = c2.coloring.flat()
    keR = oracle.all_ke(c2.mesh.nodes, c2.mesh.elements, 4, 2.1e11, 0.3, 0.1, mode=oracle.REF)
    bdR = oracle.invert_block_diag(oracle.block_diag(c2.mesh.nodeCount, c2.mesh.elements, 4,
                                                     keR, oracle.REF), c2.cons_mask, oracle.REF)
    xr, _it, _r, conv = oracle.solve_pcg(c2.mesh.nodeCount, c2.mesh.elements, 4, keR, offs,
                                         flat, c2.cons_mask, bdR, c2.F.astype(np.float64),
                                         1e-6, 20000, oracle.REF)
    assert conv and abs(max_w(x) - max_w(xr)) / abs(max_w(xr)) < 1e-4


def test_two_level_small_and_dkt(gpu_ctx, oracle):
    for wl in (workloads.plate_q4_32(), None):
        if wl is None:
            m = mesher.split_triangle_mesh(10, 10, 30, 30, jitter=0.2, seed=6)
            rng = np.random.default_rng(6)
            et = np.clip(0.1 * (1 + 0.3 * rng.standard_normal(m.elementCount)), 0.05, 0.15)
            sup = [PlateSupport("fixed", "all_edges")]
            cons = problem.identifyConstrainedDOFs(m, sup)
            F = problem.pressure_load_vector(m, 3e3).astype(np.float32)
            problem.applyBCsToRHS(F, cons)
            wl = workloads.Workload("dkt30", m, PlateMaterial(2.1e11, 0.3, 0.1,
                                                              elem_t=et.astype(np.float32)),
                                    coloring.computeElementColoringGreedy(m), sup, cons, F)
        ke, A, bd, b = fp64_operator(oracle, wl)
        import scipy.sparse.linalg as spla
        xs = spla.spsolve(A.tocsc(), b)
        for prec in (_lib.PG_PREC_FP64, _lib.PG_PREC_MIXED):
            x, info = gsolve(gpu_ctx, wl, tolerance=1e-8, max_iterations=20000, precision=prec,
                             stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=TL)
            assert info.converged
            assert rel_err(x, xs) < 1e-6


def test_two_level_fewer_iterations_than_block_jacobi(gpu_ctx, c2):
    _x, bj = gsolve(gpu_ctx, c2, tolerance=1e-6, max_iterations=20000,
                    stop_rule=_lib.PG_STOP_RELATIVE)
    _x, tl = gsolve(gpu_ctx, c2, tolerance=1e-6, max_iterations=20000,
                    stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=TL)
    assert bj.converged and tl.converged
    assert tl.iterations * 3 < bj.iterations


def test_two_level_drops_the_modes_of_constrained_parts(gpu_ctx, oracle):
    """One node per part on a clamped 6 x 6 plate: the 24 boundary parts have
    every DOF constrained, so their 72 coarse modes are zero and the device
    factorisation drops them (75 of 147 coarse DOFs kept); the solve still
    meets the error bar against the direct solve, in FP64 and mixed
    precision."""
    wl = workloads.plate_q4(6, seed=1, edges="fixed", pressure=1e3, n_point_loads=0, name="q4_6")
    ke, A, bd, b = fp64_operator(oracle, wl)
    import scipy.sparse.linalg as spla
    xs = spla.spsolve(A.tocsc(), b)
    for prec in (_lib.PG_PREC_FP64, _lib.PG_PREC_MIXED):
        x, info = gsolve(gpu_ctx, wl, tolerance=1e-10, max_iterations=2000, precision=prec,
                         stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=TL, ctas=49)
        assert info.ctas == 49 and info.coarse_dim == 3 * (49 - 24)
        assert info.converged and rel_err(x, xs) < 1e-6
