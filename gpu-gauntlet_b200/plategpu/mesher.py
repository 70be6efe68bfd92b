"""Structured plate meshes (host side, numpy).

generateRectangularMesh mirrors src/lib/plate/mesher.ts:364-439 (node
numbering j*(nx+1)+i, float32 coordinates i*dx, CCW quads 0-1-2-3, boundary
list bottom, right, top, left).  The split-triangle mesh is the DKT workload's
geometry: every quad of the same grid split in two along alternating
diagonals, interior nodes jittered.
"""
from __future__ import annotations

import math

import numpy as np

from .types import PlateMesh


def rectangular_mesh_dims(width: float, height: float, targetSize: float = 0.5):
    """mesher.ts:370-371."""
    return max(2, math.ceil(width / targetSize)), max(2, math.ceil(height / targetSize))


def rectangular_mesh_nxny(width: float, height: float, nx: int, ny: int) -> PlateMesh:
    """The body of generateRectangularMesh for explicit nx, ny."""
    dx = width / nx
    dy = height / ny
    nodesX = nx + 1
    i = np.arange(nx + 1, dtype=np.float64)
    j = np.arange(ny + 1, dtype=np.float64)
    nodes = np.empty((ny + 1, nx + 1, 2), np.float32)
    nodes[:, :, 0] = (i * dx)[None, :].astype(np.float32)
    nodes[:, :, 1] = (j * dy)[:, None].astype(np.float32)
    jj, ii = np.meshgrid(np.arange(ny, dtype=np.int64), np.arange(nx, dtype=np.int64),
                         indexing="ij")
    n0 = jj * nodesX + ii
    el = np.stack([n0, n0 + 1, n0 + nodesX + 1, n0 + nodesX], axis=-1).reshape(-1)
    b = [np.arange(nx + 1), np.arange(1, ny + 1) * nodesX + nx,
         ny * nodesX + np.arange(nx - 1, -1, -1), np.arange(ny - 1, 0, -1) * nodesX]
    boundary = np.concatenate(b)
    return PlateMesh(nodes=nodes.reshape(-1), elements=el.astype(np.uint32),
                     boundaryNodes=boundary.astype(np.uint32), nodeCount=(nx + 1) * (ny + 1),
                     elementCount=nx * ny, nodesPerElement=4, gridNx=nx, gridNy=ny)


def generateRectangularMesh(width: float, height: float, targetSize: float = 0.5) -> PlateMesh:
    """mesher.ts:364-439."""
    nx, ny = rectangular_mesh_dims(width, height, targetSize)
    return rectangular_mesh_nxny(width, height, nx, ny)


def split_triangle_mesh(width: float, height: float, nx: int, ny: int, jitter: float = 0.0,
                        seed: int = 0) -> PlateMesh:
    """nx*ny quads, each split into two triangles along alternating diagonals
    ((i + j) even: 0-2 diagonal, odd: 1-3 diagonal), both CCW.  Interior
    nodes move by U(-jitter*h, +jitter*h) in x and y (h = element size),
    drawn from ``seed``.  gridNx is 0: the reference treats such meshes as
    unstructured and colours them greedily (solver.ts:513-516)."""
    base = rectangular_mesh_nxny(width, height, nx, ny)
    xy = base.nodes.astype(np.float64).reshape(ny + 1, nx + 1, 2)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        hx, hy = width / nx, height / ny
        d = rng.uniform(-jitter, jitter, size=(ny - 1, nx - 1, 2))
        xy[1:-1, 1:-1, 0] += d[..., 0] * hx
        xy[1:-1, 1:-1, 1] += d[..., 1] * hy
    q = base.elements.reshape(ny, nx, 4).astype(np.int64)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    even = ((ii + jj) % 2 == 0)[..., None]
    t1 = np.where(even, q[..., [0, 1, 2]], q[..., [0, 1, 3]])
    t2 = np.where(even, q[..., [0, 2, 3]], q[..., [1, 2, 3]])
    tri = np.stack([t1, t2], axis=2).reshape(-1)
    return PlateMesh(nodes=xy.reshape(-1).astype(np.float32), elements=tri.astype(np.uint32),
                     boundaryNodes=base.boundaryNodes, nodeCount=base.nodeCount,
                     elementCount=2 * nx * ny, nodesPerElement=3, gridNx=0, gridNy=0)


def getElementCoords(mesh: PlateMesh, elementIndex: int) -> np.ndarray:
    """mesher.ts:448-463."""
    npe = mesh.nodesPerElement
    idx = mesh.elements[elementIndex * npe:(elementIndex + 1) * npe].astype(np.int64)
    return mesh.nodes.reshape(-1, 2)[idx].reshape(-1).copy()
