"""Nodal bending moments on the GPU (pg_moments, pg_plan_moments_device)
against the oracle's restatement of computeMoments (postprocess.ts:40-264):
FP64 oracle to 1e-12 and reference-precision oracle to 1e-6, relative to
the largest moment, for Q4 and DKT meshes."""
import numpy as np
import pytest

from plategpu import _lib, computeMoments, mesher, workloads
from plategpu.types import PlateMaterial

pytestmark = pytest.mark.gpu


def solution(oracle, wl):
    m, mat = wl.mesh, wl.material
    ke = oracle.all_ke(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t,
                       elem_t=mat.elem_t, mode=oracle.FP64)
    x, _ = oracle.truth_solve(m.nodeCount, m.elements, m.nodesPerElement, ke, wl.cons_mask, wl.F)
    return x


def check(gpu_ctx, oracle, wl, x):
    m, mat = wl.mesh, wl.material
    pr = _lib.Problem(m, mat, wl.coloring, wl.F, wl.cons_mask)
    got = gpu_ctx.moments(pr, x)
    for mode, tol in ((oracle.FP64, 1e-12), (oracle.REF, 1e-6)):
        want = oracle.moments(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t, x, mode)
        scale = max(np.abs(w).max() for w in want)
        for g, w in zip(got, want):
            assert np.abs(g - w).max() <= tol * scale
    return got


def test_moments_q4(gpu_ctx, oracle):
    wl = workloads.plate_q4_32()
    x = solution(oracle, wl)
    got = check(gpu_ctx, oracle, wl, x)
    mir = computeMoments(wl.mesh, x, wl.material)
    assert mir["Mx"].dtype == np.float32
    assert np.allclose(mir["Mx"], got[0].astype(np.float32))


def test_moments_dkt_with_a_degenerate_triangle(gpu_ctx, oracle):
    m = mesher.split_triangle_mesh(10, 10, 12, 12, jitter=0.2, seed=3)
    wl = workloads.Workload("dkt12", m, PlateMaterial(2.1e11, 0.3, 0.1), None, [], set(),
                            np.zeros(3 * m.nodeCount, np.float32))
    rng = np.random.default_rng(2)
    x = rng.standard_normal(3 * m.nodeCount) * 1e-3
    check(gpu_ctx, oracle, wl, x)
    # collapse one triangle: the reference skips it in the averages
    el = m.elements.reshape(-1, 3)
    nodes = m.nodes.copy().reshape(-1, 2)
    a, b, c = el[5]
    nodes[c] = nodes[a] + 0.5 * (nodes[b] - nodes[a])
    m2 = type(m)(**{**m.__dict__, "nodes": nodes.reshape(-1)})
    wl2 = workloads.Workload("dkt12d", m2, wl.material, None, [], set(), wl.F)
    check(gpu_ctx, oracle, wl2, x)


def test_plan_moments_device(gpu_ctx, oracle):
    torch = pytest.importorskip("torch")
    wl = workloads.plate_q4_32()
    x = solution(oracle, wl)
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    plan = gpu_ctx.plan(pr, _lib.make_options())
    xd = torch.from_numpy(x).cuda()
    md = torch.zeros(3 * wl.mesh.nodeCount, dtype=torch.float64, device="cuda")
    gpu_ctx._check(gpu_ctx.L.pg_plan_moments_device(plan.h, xd.data_ptr(), md.data_ptr()))
    torch.cuda.synchronize()
    got = md.cpu().numpy().reshape(3, -1)
    host = gpu_ctx.moments(pr, x)
    for g, h in zip(got, host):
        assert np.array_equal(g, h)
    plan.close()
