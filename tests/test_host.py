"""Host-side mirrors (mesher, colouring, supports, loads, workloads) vs the oracle."""
import numpy as np
import pytest

from plategpu import coloring as col
from plategpu import mesher, problem, workloads
from plategpu.types import PlateLoad, PlateSupport


@pytest.mark.parametrize("w,h,target", [(10, 10, 2.0), (10, 10, 0.28), (7.5, 3.0, 0.4),
                                         (10, 10, 10 / 141)])
def test_rectangular_mesh_matches_oracle(oracle, w, h, target):
    m = mesher.generateRectangularMesh(w, h, target)
    nx, ny = oracle.rect_dims(w, h, target)
    assert (m.gridNx, m.gridNy) == (nx, ny)
    nodes, el, bnd = oracle.rect_mesh(w, h, nx, ny)
    np.testing.assert_array_equal(m.nodes, nodes)
    np.testing.assert_array_equal(m.elements, el)
    np.testing.assert_array_equal(m.boundaryNodes, bnd)


def test_dof_counts_of_workload_meshes():
    assert 3 * mesher.rectangular_mesh_nxny(10, 10, 32, 32).nodeCount == 3267
    assert 3 * mesher.rectangular_mesh_nxny(10, 10, 141, 141).nodeCount == 60492
    t = mesher.split_triangle_mesh(10, 10, 200, 200, jitter=0.2, seed=1)
    assert 3 * t.nodeCount == 121203 and t.elementCount == 80000


def test_structured_coloring_matches_oracle(oracle):
    m = mesher.rectangular_mesh_nxny(10, 10, 9, 6)
    c = col.computeElementColoring(m)
    ec, flat, counts = oracle.color_structured(m.elementCount, m.gridNx)
    np.testing.assert_array_equal(c.elementColors, ec)
    np.testing.assert_array_equal(np.concatenate(c.colors), flat)
    assert col.verifyColoring(m, c)


def test_greedy_coloring_matches_oracle(oracle):
    m = mesher.split_triangle_mesh(10, 10, 11, 9, jitter=0.2, seed=3)
    c = col.computeElementColoringGreedy(m)
    ec, flat, counts = oracle.color_greedy(m.nodeCount, m.elementCount, 3, m.elements)
    np.testing.assert_array_equal(c.elementColors, ec)
    np.testing.assert_array_equal(np.concatenate(c.colors), flat)
    assert col.verifyColoring(m, c)


def test_constrained_dofs_match_oracle(oracle):
    m = mesher.rectangular_mesh_nxny(10, 10, 8, 8)
    sups = [PlateSupport("pinned", "all_edges"), PlateSupport("fixed", 40),
            PlateSupport("roller", 12)]
    got = problem.constrained_mask(3 * m.nodeCount, problem.identifyConstrainedDOFs(m, sups))
    ref = oracle.constrained(m.nodeCount, [(s.type, s.location) for s in sups], m.boundaryNodes)
    np.testing.assert_array_equal(got, ref)


def test_load_vector_matches_oracle(oracle):
    m = mesher.rectangular_mesh_nxny(10, 10, 16, 16)
    rng = np.random.default_rng(0)
    loads = [PlateLoad((float(a), float(b)), float(c)) for a, b, c in
             zip(rng.uniform(0, 10, 9), rng.uniform(0, 10, 9), rng.uniform(1e3, 1e4, 9))]
    loads.append(PlateLoad((5.0, 5.0), 1234.5))
    loads.append(PlateLoad((5.0, 5.0), 0.1))  # accumulates in float32 at the same node
    F = problem.buildLoadVector(m, loads)
    Fo = oracle.load_vector(m.nodes, [(l.position, l.magnitude) for l in loads], 0)
    np.testing.assert_array_equal(F.astype(np.float64), Fo)


def test_pressure_load_total():
    m = mesher.split_triangle_mesh(10, 10, 20, 20, jitter=0.2, seed=7)
    F = problem.pressure_load_vector(m, 3e3)
    assert abs(F.sum() - 3e3 * 100.0) < 1e-6 * 3e5


@pytest.mark.parametrize("name,ndof", [("plate_q4_32", 3267), ("plate_q4_141", 60492)])
def test_workload_shapes(name, ndof):
    wl = workloads.WORKLOADS[name]()
    assert wl.n_dof == ndof
    assert wl.F.dtype == np.float32 and np.all(wl.F[wl.cons_mask != 0] == 0)
    assert col.verifyColoring(wl.mesh, wl.coloring)
    wl2 = workloads.WORKLOADS[name]()
    np.testing.assert_array_equal(wl.F, wl2.F)  # seeded


def test_q4_141_columns_and_loads():
    wl = workloads.plate_q4_141()
    cols = [s for s in wl.supports if s.location != "all_edges"]
    assert len(cols) == 16
    assert len(wl.point_loads) == 32
    assert all(1e3 <= m <= 1e4 for _p, m in wl.point_loads)


def test_dkt_workload_thickness_field():
    wl = workloads.plate_dkt_200()
    t = wl.material.elem_t
    assert t.size == 80000 and t.min() >= 0.05 and t.max() <= 0.15
    assert 0.08 < float(t.mean()) < 0.12 and t.std() > 0.005
    assert wl.n_dof == 121203
    assert col.verifyColoring(wl.mesh, wl.coloring)


def test_solver_options_are_checked_before_any_device_work():
    from plategpu import PlateGPUError, solveGPU
    from plategpu.types import GPUSolverOptions
    wl = workloads.plate_q4(4, 0)
    for bad in (dict(preconditioner="multigrid"), dict(smoother="gauss-seidel"),
                dict(precision="fp16"), dict(stopRule="absolute")):
        with pytest.raises(PlateGPUError, match="unknown"):
            solveGPU(wl.mesh, wl.material, wl.coloring, wl.F, wl.constrainedDOFs,
                     GPUSolverOptions(**bad))


def test_postprocess_host_helpers():
    from plategpu import extractVerticalDisplacements, findMaxDisplacement, findMaxMoments
    x = np.array([1, 9, 9, -3, 9, 9, 3, 9, 9], np.float32)
    w = extractVerticalDisplacements(x, 3)
    assert w.tolist() == [1, -3, 3]
    nodes = np.array([0, 0, 1, 0, 2, 0], np.float32)
    m = findMaxDisplacement(w, nodes)
    assert m == {"maxW": -3.0, "nodeIndex": 1, "x": 1.0, "y": 0.0}  # first of equal magnitudes
    mm = findMaxMoments([1, -5, 2], [0.5, 0.25, -0.75], [3, 3, -3])
    assert mm == {"maxMx": -5.0, "maxMy": -0.75, "maxMxy": 3.0}


def test_oracle_moments_of_a_pure_bending_field(oracle):
    """theta_y = c x (so kx = c) and theta_x = -d y (ky = d) on a rectangle:
    every element carries the same curvatures, so every node gets
    Mx = D (c + nu d), My = D (d + nu c), Mxy = 0, in both modes."""
    m = mesher.rectangular_mesh_nxny(4, 3, 8, 6)
    xy = m.nodes.reshape(-1, 2).astype(np.float64)
    c, d = 1e-3, -2e-3
    x = np.zeros(3 * m.nodeCount)
    x[1::3] = -d * xy[:, 1]
    x[2::3] = c * xy[:, 0]
    E, nu, t = 2.1e11, 0.3, 0.1
    D = E * t ** 3 / (12 * (1 - nu ** 2))
    for mode in (oracle.FP64, oracle.REF):
        Mx, My, Mxy = oracle.moments(m.nodes, m.elements, 4, E, nu, t, x, mode)
        assert np.allclose(Mx, D * (c + nu * d), rtol=1e-6)
        assert np.allclose(My, D * (d + nu * c), rtol=1e-6)
        assert np.abs(Mxy).max() < 1e-6 * abs(D * c)


def test_unstructured_mesh_colouring_and_plans(oracle):
    """A plate with holes (Delaunay triangles, shuffled node numbers): greedy
    colouring agrees with the oracle and is valid, and the host partition
    keeps its invariants at several part counts and both halo widths."""
    import unstructured as U
    from plategpu import _lib

    wl = U.workload(h=0.2)
    m = wl.mesh
    el = m.elements.reshape(-1, 3)
    xy = m.nodes.reshape(-1, 2).astype(np.float64)
    d = xy[el]
    area2 = (d[:, 1, 0] - d[:, 0, 0]) * (d[:, 2, 1] - d[:, 0, 1]) - \
        (d[:, 2, 0] - d[:, 0, 0]) * (d[:, 1, 1] - d[:, 0, 1])
    assert (area2 > 0).all()
    assert col.verifyColoring(m, wl.coloring)
    ec, flat, _counts = oracle.color_greedy(m.nodeCount, m.elementCount, 3, m.elements)
    np.testing.assert_array_equal(ec, wl.coloring.elementColors)
    np.testing.assert_array_equal(np.concatenate(wl.coloring.colors), flat)
    pr = _lib.Problem(m, wl.material, wl.coloring, wl.F, wl.cons_mask)
    for ctas in (5, 37, 148):
        for rings in (1, 2):
            st = _lib.plan_inspect(pr, ctas, rings=rings)
            assert st["violations"] == 0 and st["parts"] == ctas and st["recolored"] == 0


def test_reference_dkt_zero_mode_at_third_vertex_nodes(oracle):
    """The reference's DKT element (element.ts:642-943 as written) leaves a
    zero-energy mode at every free node that is the third vertex of all its
    triangles; the test meshes rotate vertex lists so that none is."""
    import unstructured as U

    for rotate in (False, True):
        wl = U.workload(h=0.5, rotate=rotate)
        m, mat = wl.mesh, wl.material
        el = m.elements.reshape(-1, 3)
        front = np.zeros(m.nodeCount, bool)
        front[el[:, 0]] = True
        front[el[:, 1]] = True
        free = ~wl.cons_mask.reshape(-1, 3).all(1)
        third_only = int((~front & free).sum())
        ke = oracle.all_ke(m.nodes, m.elements, 3, mat.E, mat.nu, mat.t, elem_t=mat.elem_t, mode=oracle.FP64)
        w = np.linalg.eigvalsh(oracle.assemble(m.nodeCount, m.elements, 3, ke, wl.cons_mask).toarray())
        zero = int((np.abs(w) < 1e-14 * w[-1]).sum())
        assert zero == third_only
        assert (third_only > 0) == (not rotate)
