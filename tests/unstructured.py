"""Unstructured triangle meshes for the tests: a plate with holes,
triangulated by Delaunay over boundary, hole and interior points, with the
node numbering shuffled.

The reference meshes such plates with a constrained Delaunay triangulation
(mesher-unstructured.ts:36-76, through the poly2tri package).  The mesher is
not on the solver's path; these meshes only stand in for its output: CCW
triangles, irregular node valence, holes, and node numbers with no spatial
order, fed to the same kernels through greedy colouring
(coloring.ts:92-177).
"""
import numpy as np
from scipy.spatial import Delaunay

from plategpu import coloring, problem
from plategpu.types import PlateMaterial, PlateMesh, PlateSupport
from plategpu.workloads import Workload


def _circle(cx, cy, r, h):
    n = max(8, int(np.ceil(2 * np.pi * r / h)))
    a = 2 * np.pi * np.arange(n) / n
    return np.stack([cx + r * np.cos(a), cy + r * np.sin(a)], 1)


def _rotate_vertex_order(tri, n, rng):
    """Cyclic rotations of each triangle's vertex list (orientation kept)
    such that every node is the first or second vertex of at least one of
    its triangles.  The reference's DKT element (element.ts:642-943, B built
    from the derivatives in L1 and L2) gives a node that is the third
    vertex of all its triangles a zero-energy mode, so such a mesh is
    singular under the reference's own operator."""
    tri = tri.copy()
    shift = rng.integers(0, 3, len(tri))
    for k in range(3):
        sel = shift == k
        tri[sel] = np.roll(tri[sel], k, axis=1)
    for _ in range(100):
        front = np.zeros(n, bool)
        front[tri[:, 0]] = True
        front[tri[:, 1]] = True
        bad = np.flatnonzero(~front)
        if len(bad) == 0:
            return tri
        for v in bad:  # move v to the front of one of its triangles
            t = np.flatnonzero(tri[:, 2] == v)[0]
            tri[t] = tri[t][[2, 0, 1]]
    raise RuntimeError("vertex order not settled")


def plate_with_holes(width=10.0, height=10.0, h=0.25, holes=((6.0, 4.0, 1.5), (2.5, 7.0, 0.8)),
                     seed=3, shuffle=True, rotate=True):
    """PlateMesh (3 nodes per element) of a width x height plate with
    circular holes (cx, cy, r), target edge length h.  Interior points sit
    on an offset grid with a small seeded jitter, as the reference's Steiner
    points do (mesher-unstructured.ts:86-130).  Returns (mesh, outer, hole)
    where outer / hole are the node ids on the outer and hole boundaries.
    rotate=False keeps the triangulation's own vertex order."""
    rng = np.random.default_rng(seed)
    nx, ny = int(np.ceil(width / h)), int(np.ceil(height / h))
    xs, ys = np.linspace(0, width, nx + 1), np.linspace(0, height, ny + 1)
    outer = np.concatenate([np.stack([xs, np.zeros_like(xs)], 1),
                            np.stack([np.full(ny - 1, width), ys[1:-1]], 1),
                            np.stack([xs[::-1], np.full_like(xs, height)], 1),
                            np.stack([np.zeros(ny - 1), ys[-2:0:-1]], 1)])
    rings = [_circle(cx, cy, r, h) for cx, cy, r in holes]
    pts = []
    for j in range(1, ny):
        off = 0.5 * h if j % 2 else 0.0
        for i in range(1, nx):
            x, y = i * h + off, j * h
            if x > width - 0.3 * h or y > height - 0.3 * h:
                continue
            if any(np.hypot(x - cx, y - cy) < r + 0.5 * h for cx, cy, r in holes):
                continue
            pts.append((x, y))
    inner = np.asarray(pts) + rng.uniform(-0.15 * h, 0.15 * h, (len(pts), 2))
    P = np.concatenate([outer] + rings + [inner])
    n_outer, n_hole = len(outer), sum(len(r) for r in rings)
    tri = Delaunay(P).simplices
    cen = P[tri].mean(1)
    keep = np.ones(len(tri), bool)
    for cx, cy, r in holes:
        keep &= np.hypot(cen[:, 0] - cx, cen[:, 1] - cy) > r
    tri = tri[keep]
    # counter-clockwise, as the reference's triangles are
    d = P[tri]
    area2 = (d[:, 1, 0] - d[:, 0, 0]) * (d[:, 2, 1] - d[:, 0, 1]) - \
        (d[:, 2, 0] - d[:, 0, 0]) * (d[:, 1, 1] - d[:, 0, 1])
    tri[area2 < 0] = tri[area2 < 0][:, [0, 2, 1]]
    used = np.unique(tri)
    assert len(used) == len(P)  # every point is a vertex of a kept triangle
    if rotate:
        tri = _rotate_vertex_order(tri, len(P), rng)
    perm = rng.permutation(len(P)) if shuffle else np.arange(len(P))  # old -> new id
    nodes = np.empty_like(P)
    nodes[perm] = P
    tri = perm[tri]
    outer_ids = perm[:n_outer]
    hole_ids = perm[n_outer:n_outer + n_hole]
    mesh = PlateMesh(nodes=nodes.astype(np.float32).ravel(), elements=tri.astype(np.uint32).ravel(),
                     boundaryNodes=np.concatenate([outer_ids, hole_ids]).astype(np.uint32),
                     nodeCount=len(P), elementCount=len(tri), nodesPerElement=3)
    return mesh, outer_ids, hole_ids


def workload(h=0.25, seed=3, q=4e3, t=0.1, rotate=True):
    """Clamped outer edges, free hole edges, uniform pressure q plus two
    point loads; per-element thickness varying smoothly across the plate."""
    m, outer, _hole = plate_with_holes(h=h, seed=seed, rotate=rotate)
    sup = [PlateSupport("fixed", int(k)) for k in outer]
    cons = problem.identifyConstrainedDOFs(m, sup)
    F64 = problem.pressure_load_vector(m, q)
    xy = m.nodes.reshape(-1, 2).astype(np.float64)
    for px, py, P in ((3.0, 3.0, 5e3), (7.5, 8.0, 8e3)):
        k = int(np.argmin(np.hypot(xy[:, 0] - px, xy[:, 1] - py)))
        F64[3 * k] += P
    F = F64.astype(np.float32)
    problem.applyBCsToRHS(F, cons)
    el = m.elements.reshape(-1, 3)
    cen = xy[el].mean(1)
    et = (t * (1.0 + 0.3 * np.sin(0.6 * cen[:, 0]) * np.cos(0.4 * cen[:, 1]))).astype(np.float32)
    mat = PlateMaterial(2.1e11, 0.3, t, elem_t=et)
    return Workload("plate_holes_dkt", m, mat, coloring.computeElementColoringGreedy(m), sup, cons, F)
