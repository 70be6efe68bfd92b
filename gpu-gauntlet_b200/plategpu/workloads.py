"""Seeded synthetic plate workloads.

Every workload is a 10 m x 10 m plate, E = 2.1e11 Pa, nu = 0.3, shear
correction 5/6 (fixed in the element, element.ts:235), built through the
host mirrors of the reference's mesher / colouring / support / load
functions.  Loads are a uniform pressure (as nodal equivalent loads) plus
point loads at seeded nodes, rounded once to the float32 F of the solver
interface, with the constrained entries zeroed (applyBCsToRHS).

  plate_q4_32      32x32 Q4 (3,267 DOF), all edges clamped, 1 kPa + 4 point
                   loads U(1,10) kN at seeded interior nodes.
  plate_q4_141     141x141 Q4 (60,492 DOF), edges simply supported (w = 0)
                   plus w = 0 at a seeded 4x4 grid of interior column nodes,
                   5 kPa + 32 point loads U(1,10) kN at seeded nodes.
  batch_uneven     256 independent plates of uneven size, element type,
                   material, supports and random-field loads (see its
                   docstring); a list of workloads for the batched solver.
  plate_dkt_200    200x200 quads split into 80,000 DKT triangles along
                   alternating diagonals (121,203 DOF), interior nodes
                   jittered U(-0.2h, 0.2h), thickness 0.1(1 + 0.3 g) clipped
                   to [0.05, 0.15] with g a squared-exponential Gaussian
                   random field (length-scale 2 m), clamped edges, 3 kPa.
  plate_q4_400     400x400 Q4 (482,403 DOF), as plate_q4_141 otherwise: too
                   large for the persistent kernel's shared memory.
  plate_holes_dkt  an unstructured DKT plate with two circular holes
                   (Delaunay triangles, shuffled node numbers; 6,615 nodes at
                   the default h = 0.12): clamped outer edges, free hole
                   edges, 4 kPa + two point loads, smoothly varying
                   thickness.  Stands in for the reference's constrained-
                   Delaunay meshes (mesher-unstructured.ts:36-76).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import coloring as _col
from . import mesher as _mesh
from . import problem as _prob
from .types import ElementColoring, PlateMaterial, PlateMesh, PlateSupport

WIDTH = 10.0
E_STEEL = 2.1e11
NU = 0.3
T_PLATE = 0.1


@dataclass
class Workload:
    name: str
    mesh: PlateMesh
    material: PlateMaterial
    coloring: ElementColoring
    supports: List[PlateSupport]
    constrainedDOFs: set
    F: np.ndarray  # float32, BCs applied
    point_loads: list = field(default_factory=list)
    description: str = ""

    @property
    def n_dof(self) -> int:
        return self.mesh.nodeCount * 3

    @property
    def cons_mask(self) -> np.ndarray:
        return _prob.constrained_mask(self.n_dof, self.constrainedDOFs)


def _finish_loads(mesh, pressure, point_nodes, point_mags, constrainedDOFs):
    F = _prob.pressure_load_vector(mesh, pressure)
    xy = mesh.nodes.reshape(-1, 2)
    loads = []
    for n, m in zip(point_nodes, point_mags):
        F[3 * int(n)] += float(m)
        loads.append(((float(xy[n, 0]), float(xy[n, 1])), float(m)))
    F32 = F.astype(np.float32)
    _prob.applyBCsToRHS(F32, constrainedDOFs)
    return F32, loads


def _interior_nodes(nx, ny):
    jj, ii = np.meshgrid(np.arange(1, ny), np.arange(1, nx), indexing="ij")
    return (jj * (nx + 1) + ii).reshape(-1)


def plate_q4(nx: int, seed: int, edges: str = "fixed", pressure: float = 1e3,
             n_point_loads: int = 4, column_grid: int = 0, t: float = T_PLATE,
             E: float = E_STEEL, nu: float = NU, name: Optional[str] = None) -> Workload:
    """Structured nx x nx Q4 Mindlin plate with seeded loads and columns."""
    rng = np.random.default_rng(seed)
    mesh = _mesh.rectangular_mesh_nxny(WIDTH, WIDTH, nx, nx)
    supports = [PlateSupport(edges, "all_edges")]
    if column_grid:
        # a k x k grid of interior column nodes, each grid line shifted by a
        # seeded offset of up to 2 elements
        base = [round((a + 1) * nx / (column_grid + 1)) for a in range(column_grid)]
        off_i = rng.integers(-2, 3, size=column_grid)
        off_j = rng.integers(-2, 3, size=column_grid)
        for a in range(column_grid):
            for b in range(column_grid):
                i = int(np.clip(base[a] + off_i[a], 1, nx - 1))
                j = int(np.clip(base[b] + off_j[b], 1, nx - 1))
                supports.append(PlateSupport("pinned", j * (nx + 1) + i))
    cons = _prob.identifyConstrainedDOFs(mesh, supports)
    interior = _interior_nodes(nx, nx)
    free_w = np.array([n for n in interior if 3 * int(n) not in cons])
    nodes = rng.choice(free_w, size=n_point_loads, replace=False)
    mags = rng.uniform(1e3, 1e4, size=n_point_loads)
    F, loads = _finish_loads(mesh, pressure, nodes, mags, cons)
    return Workload(name=name or f"plate_q4_{nx}", mesh=mesh,
                    material=PlateMaterial(E=E, nu=nu, t=t),
                    coloring=_col.computeElementColoring(mesh), supports=supports,
                    constrainedDOFs=cons, F=F, point_loads=loads)


def plate_q4_32(seed: int = 1) -> Workload:
    return plate_q4(32, seed, edges="fixed", pressure=1e3, n_point_loads=4,
                    name="plate_q4_32")


def plate_q4_141(seed: int = 2) -> Workload:
    return plate_q4(141, seed, edges="pinned", pressure=5e3, n_point_loads=32, column_grid=4,
                    name="plate_q4_141")


def plate_q4_400(seed: int = 4) -> Workload:
    """400 x 400 Q4 (160,801 nodes, 482,403 DOF), loads and supports as
    plate_q4_141: past the persistent kernel's shared-memory capacity, so
    the solver runs its global-memory path."""
    return plate_q4(400, seed, edges="pinned", pressure=5e3, n_point_loads=32, column_grid=4,
                    name="plate_q4_400")


def grf_squared_exponential(nx: int, ny: int, h: float, length: float,
                            rng: np.random.Generator) -> np.ndarray:
    """Zero-mean, unit-variance Gaussian random field with squared-
    exponential covariance exp(-d^2 / (2 l^2)) on an (ny+1) x (nx+1) node
    grid of spacing h, sampled spectrally on a periodic grid padded by
    4 l so that the wrap-around correlation is negligible."""
    pad = int(np.ceil(4 * length / h))
    Mx, My = nx + 1 + pad, ny + 1 + pad
    kx = 2 * np.pi * np.fft.fftfreq(Mx, d=h)
    ky = 2 * np.pi * np.fft.fftfreq(My, d=h)
    K2 = ky[:, None] ** 2 + kx[None, :] ** 2
    spec = np.exp(-0.5 * length ** 2 * K2)
    noise = rng.standard_normal((My, Mx))
    field = np.real(np.fft.ifft2(np.fft.fft2(noise) * np.sqrt(spec)))
    field = field[: ny + 1, : nx + 1]
    return (field - field.mean()) / field.std()


def plate_dkt_200(seed: int = 3, n: int = 200) -> Workload:
    rng = np.random.default_rng(seed)
    mesh = _mesh.split_triangle_mesh(WIDTH, WIDTH, n, n, jitter=0.2,
                                     seed=int(rng.integers(1 << 31)))
    g_nodes = grf_squared_exponential(n, n, WIDTH / n, 2.0, rng).reshape(-1)
    el = mesh.elements.astype(np.int64).reshape(-1, 3)
    g_elem = g_nodes[el].mean(axis=1)
    elem_t = np.clip(T_PLATE * (1 + 0.3 * g_elem), 0.05, 0.15).astype(np.float32)
    supports = [PlateSupport("fixed", "all_edges")]
    cons = _prob.identifyConstrainedDOFs(mesh, supports)
    F, loads = _finish_loads(mesh, 3e3, [], [], cons)
    return Workload(name=f"plate_dkt_{n}", mesh=mesh,
                    material=PlateMaterial(E=E_STEEL, nu=NU, t=T_PLATE, elem_t=elem_t),
                    coloring=_col.computeElementColoringGreedy(mesh), supports=supports,
                    constrainedDOFs=cons, F=F, point_loads=loads)


def _edge_supports(mesh: PlateMesh, kinds) -> List[PlateSupport]:
    """One support per boundary node: kinds[e] ('fixed' clamped or 'pinned'
    simply supported) for the left, right, bottom and top edge; a corner
    takes the stronger of its two edges."""
    xy = mesh.nodes.reshape(-1, 2)
    lo, hi = xy.min(axis=0), xy.max(axis=0)
    tol = 1e-6 * max(1.0, float(np.max(hi - lo)))
    on = [np.abs(xy[:, 0] - lo[0]) < tol, np.abs(xy[:, 0] - hi[0]) < tol,
          np.abs(xy[:, 1] - lo[1]) < tol, np.abs(xy[:, 1] - hi[1]) < tol]
    kind = {}
    for e in range(4):
        for n in np.nonzero(on[e])[0].tolist():
            if kind.get(n) != "fixed":
                kind[n] = kinds[e]
    return [PlateSupport(k, str(n)) for n, k in sorted(kind.items())]


def batch_uneven(count: int = 256, seed: int = 5, min_side: int = 16,
                 max_side: int = 256) -> List[Workload]:
    """Independent 10 m x 10 m plates of uneven sizes: elements per side
    log-uniform in [min_side, max_side]; 70% Q4 Mindlin, 30% DKT (quads
    split along alternating diagonals, interior nodes jittered U(-0.2h,
    0.2h)); thickness U(0.05, 0.3) m, E U(2e10, 2.1e11) Pa, nu U(0.2, 0.3);
    each edge clamped or simply supported at random; load a Gaussian random
    field pressure (length-scale U(0.5, 3) m, amplitude U(1, 10) kPa,
    element values from the nodal field, taken positive downward) plus 0-16
    point loads U(1, 10) kN at random interior nodes."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(min_side), np.log(max_side)))))
        dkt = rng.uniform() < 0.3
        if dkt:
            mesh = _mesh.split_triangle_mesh(WIDTH, WIDTH, n, n, jitter=0.2,
                                             seed=int(rng.integers(1 << 31)))
            coloring = _col.computeElementColoringGreedy(mesh)
        else:
            mesh = _mesh.rectangular_mesh_nxny(WIDTH, WIDTH, n, n)
            coloring = _col.computeElementColoring(mesh)
        material = PlateMaterial(E=float(rng.uniform(2e10, 2.1e11)), nu=float(rng.uniform(0.2, 0.3)),
                                 t=float(rng.uniform(0.05, 0.3)))
        kinds = ["fixed" if rng.uniform() < 0.5 else "pinned" for _ in range(4)]
        supports = _edge_supports(mesh, kinds)
        cons = _prob.identifyConstrainedDOFs(mesh, supports)
        F, loads = _random_field_load(mesh, n, cons, rng)
        out.append(Workload(name=f"batch{i}_{'dkt' if dkt else 'q4'}_{n}", mesh=mesh,
                            material=material, coloring=coloring, supports=supports,
                            constrainedDOFs=cons, F=F, point_loads=loads))
    return out


def _random_field_load(mesh: PlateMesh, n: int, cons, rng: np.random.Generator):
    """A Gaussian random field pressure on an n x n-element plate
    (squared-exponential, length-scale U(0.5, 3) m, amplitude U(1, 10) kPa,
    element values from the nodal field, q = amp (1 + g / 2) positive
    downward) plus 0-16 point loads U(1, 10) kN at random interior nodes;
    float32, BCs applied."""
    g = grf_squared_exponential(n, n, WIDTH / n, float(rng.uniform(0.5, 3.0)), rng).reshape(-1)
    amp = float(rng.uniform(1e3, 1e4))
    npe = mesh.nodesPerElement
    el = mesh.elements.astype(np.int64).reshape(-1, npe)
    q = amp * (1.0 + 0.5 * g[el].mean(axis=1))
    k = int(rng.integers(0, 17))
    interior = _interior_nodes(n, n)
    pts = rng.choice(interior, size=k, replace=False) if k else np.zeros(0, np.int64)
    return _finish_loads(mesh, q, pts, rng.uniform(1e3, 1e4, size=k), cons)


def random_field_loads(wl: Workload, count: int, seed: int) -> np.ndarray:
    """`count` seeded random-field loads of a structured n x n plate
    (plate_q4_141: the learned preconditioner's training and held-out
    loads): each a Gaussian random field pressure plus 0-16 point loads as
    in _random_field_load.  Returns float32 [count, 3 * nodeCount]."""
    n = int(round(np.sqrt(wl.mesh.elementCount)))
    if n * n != wl.mesh.elementCount or wl.mesh.nodesPerElement != 4:
        raise ValueError("random_field_loads needs a structured n x n Q4 plate")
    rng = np.random.default_rng(seed)
    out = np.empty((count, wl.n_dof), np.float32)
    for k in range(count):
        out[k] = _random_field_load(wl.mesh, n, wl.constrainedDOFs, rng)[0]
    return out


def plate_cost(w: Workload) -> float:
    """Estimated solve work of a plate: about sqrt(n) iterations over n nodes."""
    n = float(w.mesh.nodeCount)
    return n * np.sqrt(n)


def shard_lpt(costs, parts: int) -> List[List[int]]:
    """Longest-processing-time assignment of items to `parts` shards: items
    by decreasing cost (index order on ties) each go to the currently
    lightest shard (lowest index on ties).  Deterministic, so every rank
    computes the same shards."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * parts
    out: List[List[int]] = [[] for _ in range(parts)]
    for i in order:
        k = min(range(parts), key=lambda j: (load[j], j))
        out[k].append(i)
        load[k] += float(costs[i])
    return [sorted(sh) for sh in out]


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
    circular holes (cx, cy, r), target edge length h, triangulated by
    Delaunay over boundary, hole and interior points.  Interior points sit on
    an offset grid with a small seeded jitter, as the reference's Steiner
    points do (mesher-unstructured.ts:86-130).  Returns (mesh, outer, hole)
    where outer / hole are the node ids on the outer and hole boundaries.
    rotate=False keeps the triangulation's own vertex order."""
    from scipy.spatial import Delaunay

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
    if len(np.unique(tri)) != len(P):
        raise RuntimeError("a point is not a vertex of any kept triangle")
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


def plate_holes_dkt(h=0.12, seed=3, q=4e3, t=0.1, rotate=True) -> Workload:
    """Unstructured DKT plate with holes (see the module docstring)."""
    m, outer, _hole = plate_with_holes(h=h, seed=seed, rotate=rotate)
    sup = [PlateSupport("fixed", int(k)) for k in outer]
    cons = _prob.identifyConstrainedDOFs(m, sup)
    F64 = _prob.pressure_load_vector(m, q)
    xy = m.nodes.reshape(-1, 2).astype(np.float64)
    for px, py, P in ((3.0, 3.0, 5e3), (7.5, 8.0, 8e3)):
        k = int(np.argmin(np.hypot(xy[:, 0] - px, xy[:, 1] - py)))
        F64[3 * k] += P
    F = F64.astype(np.float32)
    _prob.applyBCsToRHS(F, cons)
    el = m.elements.reshape(-1, 3)
    cen = xy[el].mean(1)
    et = (t * (1.0 + 0.3 * np.sin(0.6 * cen[:, 0]) * np.cos(0.4 * cen[:, 1]))).astype(np.float32)
    mat = PlateMaterial(2.1e11, 0.3, t, elem_t=et)
    return Workload("plate_holes_dkt", m, mat, _col.computeElementColoringGreedy(m), sup, cons, F)


WORKLOADS = {
    "plate_q4_32": plate_q4_32,
    "plate_q4_141": plate_q4_141,
    "plate_q4_400": plate_q4_400,
    "plate_dkt_200": plate_dkt_200,
    "plate_holes_dkt": plate_holes_dkt,
}
