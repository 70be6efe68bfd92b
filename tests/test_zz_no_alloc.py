"""pg_apply_k_static: K x for callers that cannot allocate device memory.

The entry point takes device buffers for everything and keeps the element
matrices in the library's static device scratch.  Its output must match the
regular pg_apply_k (which allocates its own buffers) to the FP64 K.x
tolerance used by the other GPU tests (1e-12 relative), on consecutive calls
that reuse the same scratch with different meshes and vectors.  This file
runs last so that a failure here leaves every other test already run; it
also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from plategpu import _lib, coloring, mesher, problem
from plategpu.types import PlateMaterial, PlateSupport

pytestmark = pytest.mark.gpu


class DeviceProblem:
    """A PgProblem whose arrays live in device memory (allocated here by the
    test, not by the entry point); colour offsets stay on the host."""

    def __init__(self, torch, mesh, material, col, cons):
        offs, flat = col.flat()
        self._keep = []
        self.host_offsets = np.ascontiguousarray(offs, np.uint32)

        def dev(a):
            t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
            self._keep.append(t)
            return t.data_ptr()

        s = _lib.PgProblem()
        s.node_count = mesh.nodeCount
        s.element_count = mesh.elementCount
        s.nodes_per_element = mesh.nodesPerElement
        s.nodes = dev(mesh.nodes.astype(np.float32))
        s.elements = dev(mesh.elements.astype(np.int32))  # same bits as uint32
        s.color_count = col.colorCount
        s.color_offsets = self.host_offsets.ctypes.data
        s.elements_by_color = dev(flat.astype(np.int32))
        s.E, s.nu, s.t = material.E, material.nu, material.t
        s.elem_t = None if material.elem_t is None else dev(material.elem_t.astype(np.float32))
        s.F = None
        s.constrained = dev(np.asarray(cons, np.uint8))
        self.struct = s


def q4_case():
    m = mesher.rectangular_mesh_nxny(10, 10, 40, 40)
    cons = problem.identifyConstrainedDOFs(m, [PlateSupport("pinned", "all_edges")])
    return (m, PlateMaterial(2.1e11, 0.3, 0.1), coloring.computeElementColoring(m),
            problem.constrained_mask(3 * m.nodeCount, cons))


def dkt_case():
    m = mesher.split_triangle_mesh(10, 10, 30, 30, jitter=0.2, seed=4)
    rng = np.random.default_rng(4)
    et = rng.uniform(0.05, 0.15, m.elementCount).astype(np.float32)
    cons = problem.identifyConstrainedDOFs(m, [PlateSupport("fixed", "all_edges")])
    return (m, PlateMaterial(2.1e11, 0.3, 0.1, elem_t=et),
            coloring.computeElementColoringGreedy(m),
            problem.constrained_mask(3 * m.nodeCount, cons))


def call_static(torch, dp, x):
    L = _lib.load()
    xd = torch.from_numpy(x).cuda()
    yd = torch.full_like(xd, np.nan)  # the entry point must overwrite all of y
    msg = C.create_string_buffer(256)
    st = L.pg_apply_k_static(C.byref(dp.struct), xd.data_ptr(), yd.data_ptr(),
                             torch.cuda.current_stream().cuda_stream, msg, 256)
    assert st == _lib.PG_OK, msg.value.decode()
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def test_static_matches_apply_k_on_consecutive_calls(gpu_ctx, oracle):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(21)
    calls = [q4_case(), dkt_case(), q4_case()]
    for m, mat, col, cons in calls:
        dp = DeviceProblem(torch, m, mat, col, cons)
        hp = _lib.Problem(m, mat, col, None, cons)
        ke = oracle.all_ke(m.nodes, m.elements, m.nodesPerElement, mat.E, mat.nu, mat.t,
                           elem_t=mat.elem_t, mode=oracle.FP64)
        offs, flat = col.flat()
        for _ in range(2):
            x = rng.standard_normal(3 * m.nodeCount)
            y = call_static(torch, dp, x)
            ref = gpu_ctx.apply_k(hp, x)
            assert np.all(np.isfinite(y))
            assert rel_err(y, ref) < 1e-12
            # and directly against the FP64 oracle's K x (solver.ts:422-483)
            yo = oracle.apply_k(m.nodeCount, m.elements, m.nodesPerElement, ke, offs, flat, cons, x,
                                mode=oracle.FP64)
            assert rel_err(y, yo) < 1e-12


def test_static_rejects_overlapping_x_and_y_and_bad_offsets():
    torch = pytest.importorskip("torch")
    m, mat, col, cons = q4_case()
    dp = DeviceProblem(torch, m, mat, col, cons)
    L = _lib.load()
    n = 3 * m.nodeCount
    buf = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    msg = C.create_string_buffer(256)
    # y == x and a y that starts inside x
    for yoff in (0, 8 * (n // 2)):
        st = L.pg_apply_k_static(C.byref(dp.struct), buf.data_ptr(), buf.data_ptr() + yoff, None,
                                 msg, 256)
        assert st == _lib.PG_EINVAL and "overlap" in msg.value.decode()
    # colour offsets that start above 0, or decrease, are refused before any
    # work is queued
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    good = dp.host_offsets.copy()
    for bad in ([1] + list(good[1:]), [0, 1_000_000] + list(good[2:])):
        dp.host_offsets[:] = np.asarray(bad, np.uint32)
        st = L.pg_apply_k_static(C.byref(dp.struct), x.data_ptr(), y.data_ptr(), None, msg, 256)
        assert st == _lib.PG_EINVAL and "color_offsets" in msg.value.decode()
    dp.host_offsets[:] = good


def test_static_rejects_oversized_problem():
    torch = pytest.importorskip("torch")
    m, mat, col, cons = q4_case()
    dp = DeviceProblem(torch, m, mat, col, cons)
    dp.struct.element_count = 7282  # one more than the scratch holds
    L = _lib.load()
    x = torch.zeros(3 * m.nodeCount, dtype=torch.float64, device="cuda")
    msg = C.create_string_buffer(256)
    st = L.pg_apply_k_static(C.byref(dp.struct), x.data_ptr(), x.data_ptr(), None, msg, 256)
    assert st == _lib.PG_EINVAL
    assert "exceeds the static scratch" in msg.value.decode()
