"""GPU element stiffness, block-Jacobi set-up and K.x against the oracle.

Tolerances: FP64 GPU vs FP64 oracle to 1e-12 relative (same formulas, FMA
contraction and summation order only); FP64 GPU vs the reference-precision
oracle to the reference's own single-colour K.x tolerance, 1e-6
(gpu/single_color_test.ts:247-288).
"""
import numpy as np
import pytest

from conftest import rel_err
from plategpu import _lib, coloring, mesher, problem, workloads
from plategpu.types import PlateMaterial, PlateSupport

pytestmark = pytest.mark.gpu

E, NU = 2.1e11, 0.3


def dkt_case(n=14, seed=3, with_t=True):
    m = mesher.split_triangle_mesh(10, 10, n, n, jitter=0.2, seed=seed)
    rng = np.random.default_rng(seed)
    et = rng.uniform(0.05, 0.15, m.elementCount).astype(np.float32) if with_t else None
    mat = PlateMaterial(E, NU, 0.1, elem_t=et)
    c = coloring.computeElementColoringGreedy(m)
    cons = problem.identifyConstrainedDOFs(m, [PlateSupport("fixed", "all_edges")])
    return m, mat, c, problem.constrained_mask(3 * m.nodeCount, cons)


def q4_case(nx=12, support="pinned"):
    wl = workloads.plate_q4(nx, 1, edges=support, pressure=2e3, n_point_loads=3)
    return wl.mesh, wl.material, wl.coloring, wl.cons_mask


@pytest.mark.parametrize("kind", ["q4", "dkt"])
def test_element_stiffness(gpu_ctx, oracle, kind):
    m, mat, c, cons = q4_case() if kind == "q4" else dkt_case()
    pr = _lib.Problem(m, mat, c, None, cons)
    ke = gpu_ctx.element_stiffness(pr)
    ref64 = oracle.all_ke(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t,
                          elem_t=mat.elem_t, mode=oracle.FP64)
    assert rel_err(ke, ref64) < 1e-12
    for e in range(0, m.elementCount, 37):
        assert np.abs(ke[e] - ref64[e]).max() <= 1e-11 * np.abs(ref64[e]).max()
    refr = oracle.all_ke(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t,
                         elem_t=mat.elem_t, mode=oracle.REF)
    assert rel_err(ke, refr) < 1e-6


@pytest.mark.parametrize("kind,support", [("q4", "pinned"), ("q4", "fixed"), ("dkt", "fixed")])
def test_block_jacobi(gpu_ctx, oracle, kind, support):
    m, mat, c, cons = q4_case(support=support) if kind == "q4" else dkt_case()
    cons = cons.copy()
    cons[3 * 40 + 1] = 1  # a partially constrained interior node (theta_x only)
    pr = _lib.Problem(m, mat, c, None, cons)
    binv = gpu_ctx.block_jacobi(pr)
    npe = m.nodesPerElement
    ke = oracle.all_ke(m.nodes, m.elements, npe, mat.E, mat.nu, mat.t, elem_t=mat.elem_t,
                       mode=oracle.FP64)
    ref = oracle.invert_block_diag(oracle.block_diag(m.nodeCount, m.elements, npe, ke,
                                                     oracle.FP64), cons, oracle.FP64)
    assert rel_err(binv, ref) < 1e-11
    blocks = binv.reshape(-1, 9)
    assert np.all(blocks[np.all(cons.reshape(-1, 3) == 1, axis=1)] == np.eye(3).reshape(-1))


@pytest.mark.parametrize("kind", ["q4", "dkt"])
def test_apply_k(gpu_ctx, oracle, kind):
    m, mat, c, cons = q4_case() if kind == "q4" else dkt_case()
    pr = _lib.Problem(m, mat, c, None, cons)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(3 * m.nodeCount).astype(np.float32).astype(np.float64)
    y = gpu_ctx.apply_k(pr, x)
    npe = m.nodesPerElement
    offs, flat = c.flat()
    ke64 = oracle.all_ke(m.nodes, m.elements, npe, mat.E, mat.nu, mat.t, elem_t=mat.elem_t,
                         mode=oracle.FP64)
    y64 = oracle.apply_k(m.nodeCount, m.elements, npe, ke64, offs, flat, cons, x, oracle.FP64)
    assert rel_err(y, y64) < 1e-12
    np.testing.assert_array_equal(y[cons != 0], x[cons != 0])  # identity rows
    keR = oracle.all_ke(m.nodes, m.elements, npe, mat.E, mat.nu, mat.t, elem_t=mat.elem_t,
                        mode=oracle.REF)
    yR = oracle.apply_k(m.nodeCount, m.elements, npe, keR, offs, flat, cons, x, oracle.REF)
    assert rel_err(y, yR) < 1e-6


def test_apply_k_single_color(gpu_ctx, oracle):
    """single_color_test.ts pattern: x supported on one colour's elements."""
    m, mat, c, cons = q4_case(nx=16)
    pr = _lib.Problem(m, mat, c, None, cons)
    x = np.zeros(3 * m.nodeCount)
    el = m.elements.reshape(-1, 4)
    for e in c.colors[2]:
        x[3 * el[e].astype(np.int64)] = 1.0
    y = gpu_ctx.apply_k(pr, x)
    offs, flat = c.flat()
    ke64 = oracle.all_ke(m.nodes, m.elements, 4, mat.E, mat.nu, mat.t, mode=oracle.FP64)
    y64 = oracle.apply_k(m.nodeCount, m.elements, 4, ke64, offs, flat, cons, x, oracle.FP64)
    assert rel_err(y, y64) < 1e-12
