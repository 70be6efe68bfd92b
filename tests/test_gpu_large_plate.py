"""A plate past the persistent kernel's shared-memory capacity.

plate_q4_400 (400 x 400 Q4, 482,403 DOF) has about 1,087 nodes per part on
148 blocks, more than one block's shared memory holds.  pg_solve then runs
flexible PCG over global memory (FP32 vectors, FP64 x, dot products and
true-residual stop) instead of refusing the plate; the result must meet the
FP64 error bar (relative L2 <= 1e-6 against the sparse-LU truth) with the
reference's block Jacobi and with the smoothing steps the faster options
select.
"""
import numpy as np
import pytest

from conftest import rel_err
from plategpu import _lib, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    return workloads.plate_q4_400()


@pytest.fixture(scope="module")
def big_truth(oracle, big):
    m, mat = big.mesh, big.material
    ke = oracle.all_ke(m.nodes, m.elements, 4, mat.E, mat.nu, mat.t, mode=oracle.FP64)
    x, rel = oracle.truth_solve(m.nodeCount, m.elements, 4, ke, big.cons_mask, big.F)
    assert rel < 1e-10
    return x


@pytest.mark.parametrize("pre", [_lib.PG_PRECOND_BLOCK_JACOBI, _lib.PG_PRECOND_TWO_LEVEL])
def test_global_path_meets_the_error_bar(gpu_ctx, big, big_truth, pre):
    assert big.n_dof == 482_403
    pr = _lib.Problem(big.mesh, big.material, big.coloring, big.F, big.cons_mask)
    x, info = gpu_ctx.solve(pr, _lib.make_options(tolerance=1e-8, max_iterations=50000,
                                                  stop_rule=_lib.PG_STOP_RELATIVE, preconditioner=pre))
    assert info.global_path == 1
    assert info.converged and info.true_rel_residual < 1e-8
    assert rel_err(x, big_truth) <= 1e-6


def test_global_path_reference_stop_and_limit(gpu_ctx, big):
    pr = _lib.Problem(big.mesh, big.material, big.coloring, big.F, big.cons_mask)
    x, info = gpu_ctx.solve(pr, _lib.make_options(tolerance=1e-30, max_iterations=7))
    assert info.global_path == 1 and not info.converged and info.iterations == 7
    assert info.stop_reason == _lib.PG_STOP_MAX_ITER
    assert np.all(np.isfinite(x))
