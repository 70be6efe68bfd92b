"""Chebyshev smoother (u = a D^-1 r - b D^-1 K D^-1 r on a 2-ring ghost
halo) on the GPU, alone and inside the two-level preconditioner.

Checks: the lambda_max(D^-1 K) estimate equals the numpy power iteration
from the same start vector; FP64-checked error <= 1e-6 against the FP64
truth; the iteration count matches a numpy model of the same
preconditioner with the same coefficients (within 3% + 2: the persistent
kernel's Chronopoulos-Gear recurrence and textbook PCG agree in exact
arithmetic); the smoother cuts the two-level iteration count by a third;
and a plan made without the halo rejects the smoother.
"""
import numpy as np
import pytest

from conftest import rel_err
from plategpu import _lib, coloring, mesher, problem, workloads
from plategpu.types import PlateMaterial, PlateSupport
from test_gpu_two_level import fp64_operator, gsolve
from two_level_ref import (chebyshev2, coarse_basis, lambda_max_power, strip_partition,
                           two_level_pcg)

pytestmark = pytest.mark.gpu

TL, CHEB = _lib.PG_PRECOND_TWO_LEVEL, _lib.PG_SMOOTHER_CHEBYSHEV


@pytest.fixture(scope="module")
def c2():
    return workloads.plate_q4_141()


@pytest.mark.parametrize("precision", [_lib.PG_PREC_FP64, _lib.PG_PREC_MIXED])
def test_chebyshev_two_level_q4_141(gpu_ctx, oracle, c2, precision):
    ke, A, bd, b = fp64_operator(oracle, c2)
    import scipy.sparse.linalg as spla
    xs = spla.spsolve(A.tocsc(), b)
    x, info = gsolve(gpu_ctx, c2, tolerance=5e-6, max_iterations=20000, precision=precision,
                     stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=TL, smoother=CHEB)
    assert info.converged and info.coarse_dim == 3 * info.ctas
    assert rel_err(x, xs) < 1e-6
    lam = lambda_max_power(A, bd, c2.cons_mask)
    assert abs(info.smoother_lambda_max - lam) < 1e-6 * lam
    G = info.ctas
    part = strip_partition(c2.mesh.nodes.reshape(-1, 2).astype(np.float64), G)
    P = coarse_basis(c2.mesh.nodes.reshape(-1, 2).astype(np.float64), c2.cons_mask, part, G)
    _xm, it_m = two_level_pcg(A, b, bd, P, 5e-6, cheb=chebyshev2(info.smoother_lambda_max))
    assert abs(info.iterations - it_m) <= 0.03 * it_m + 2
    _x, plain = gsolve(gpu_ctx, c2, tolerance=5e-6, max_iterations=20000, precision=precision,
                       stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=TL)
    assert info.iterations * 3 < plain.iterations * 2


def dkt_case():
    m = mesher.split_triangle_mesh(10, 10, 30, 30, jitter=0.2, seed=8)
    rng = np.random.default_rng(8)
    et = np.clip(0.1 * (1 + 0.3 * rng.standard_normal(m.elementCount)), 0.05, 0.15)
    sup = [PlateSupport("fixed", "all_edges")]
    cons = problem.identifyConstrainedDOFs(m, sup)
    F = problem.pressure_load_vector(m, 3e3).astype(np.float32)
    problem.applyBCsToRHS(F, cons)
    return workloads.Workload("dkt30", m, PlateMaterial(2.1e11, 0.3, 0.1, elem_t=et.astype(np.float32)),
                              coloring.computeElementColoringGreedy(m), sup, cons, F)


@pytest.mark.parametrize("pc", [_lib.PG_PRECOND_BLOCK_JACOBI, TL])
def test_chebyshev_small_and_dkt(gpu_ctx, oracle, pc):
    import scipy.sparse.linalg as spla
    for wl in (workloads.plate_q4_32(), dkt_case()):
        ke, A, bd, b = fp64_operator(oracle, wl)
        xs = spla.spsolve(A.tocsc(), b)
        for prec in (_lib.PG_PREC_FP64, _lib.PG_PREC_MIXED):
            x, info = gsolve(gpu_ctx, wl, tolerance=1e-8, max_iterations=20000, precision=prec,
                             stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=pc, smoother=CHEB)
            assert info.converged
            assert rel_err(x, xs) < 1e-6
            assert 0.5 < info.smoother_lambda_max <= wl.mesh.nodesPerElement + 1e-9
        # iteration count of the FP64 solve against the numpy model
        x, info = gsolve(gpu_ctx, wl, tolerance=1e-8, max_iterations=20000,
                         stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=pc, smoother=CHEB)
        P = None
        if pc == TL:
            xy = wl.mesh.nodes.reshape(-1, 2).astype(np.float64)
            P = coarse_basis(xy, wl.cons_mask, strip_partition(xy, info.ctas), info.ctas)
        _xm, it_m = two_level_pcg(A, b, bd, P, 1e-8, cheb=chebyshev2(info.smoother_lambda_max))
        assert abs(info.iterations - it_m) <= 0.03 * it_m + 2


def test_chebyshev_needs_a_halo_plan(gpu_ctx):
    torch = pytest.importorskip("torch")
    wl = workloads.plate_q4_32()
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    plan = gpu_ctx.plan(pr, _lib.make_options())  # block Jacobi: 1-ring plan
    F = torch.from_numpy(wl.F.astype(np.float32)).cuda()
    x = torch.zeros(F.numel(), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.PlateGPUError, match="2-ring"):
        plan.solve_device(_lib.make_options(smoother=CHEB), F.data_ptr(), x.data_ptr())
    plan.close()
    plan2 = gpu_ctx.plan(pr, _lib.make_options(smoother=CHEB))
    info = plan2.solve_device(_lib.make_options(smoother=CHEB, tolerance=1e-8,
                                                stop_rule=_lib.PG_STOP_RELATIVE,
                                                max_iterations=5000), F.data_ptr(), x.data_ptr())
    assert info.converged and info.smoother_lambda_max > 0
    plan2.close()


def test_solvegpu_mirror_with_fast_options(gpu_ctx, oracle):
    """The reference-shaped entry point with the fastest measured settings."""
    from plategpu import solveGPU
    from plategpu.types import GPUSolverOptions
    wl = workloads.plate_q4_141()
    ke, A, bd, b = fp64_operator(oracle, wl)
    import scipy.sparse.linalg as spla
    xs = spla.spsolve(A.tocsc(), b)
    res = solveGPU(wl.mesh, wl.material, wl.coloring, wl.F, wl.constrainedDOFs,
                   GPUSolverOptions(tolerance=5e-6, maxIterations=5000, precision="mixed",
                                    stopRule="relative", preconditioner="two-level",
                                    smoother="chebyshev", returnFloat64=True))
    assert res.converged and res.usedGPU and res.iterations < 250
    assert rel_err(res.solution, xs) < 1e-6
