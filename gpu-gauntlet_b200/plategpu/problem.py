"""Problem definition upstream of the solver boundary (host side).

identifyConstrainedDOFs, buildLoadVector and applyBCsToRHS mirror
src/lib/plate/solver.ts:92-134, :363-392 and :400-407.  The reference API
carries only point loads; ``pressure_load_vector`` gives the nodal
equivalent of a uniform pressure (q * A_e / nodes-per-element on each
element node), the load the workloads add on top of their point loads.
"""
from __future__ import annotations

from typing import Iterable, Optional, Set

import numpy as np

from .types import DOFS_PER_NODE, PlateLoad, PlateMesh, PlateSupport


def identifyConstrainedDOFs(mesh: PlateMesh, supports: Iterable[PlateSupport]) -> Set[int]:
    """solver.ts:92-134: pinned / roller constrain w, fixed constrains
    w, theta_x, theta_y; 'all_edges' means every boundary node."""
    out: Set[int] = set()
    for s in supports:
        nodes = (mesh.boundaryNodes.tolist() if s.location == "all_edges" else [int(s.location)])
        for n in nodes:
            b = n * DOFS_PER_NODE
            if s.type in ("pinned", "roller"):
                out.add(b)
            elif s.type == "fixed":
                out.update((b, b + 1, b + 2))
            else:
                raise ValueError(f"unknown support type {s.type!r}")
    return out


def constrained_mask(n_dof: int, constrainedDOFs) -> np.ndarray:
    """Set of DOF indices -> uint8 mask (the constrainedMask buffer of
    gpu/buffers.ts:262-266, one byte per DOF)."""
    m = np.zeros(n_dof, np.uint8)
    idx = np.fromiter((int(d) for d in constrainedDOFs), dtype=np.int64)
    if idx.size:
        if idx.min() < 0 or idx.max() >= n_dof:
            raise ValueError("constrained DOF index out of range")
        m[idx] = 1
    return m


def buildLoadVector(mesh: PlateMesh, loads: Iterable[PlateLoad]) -> np.ndarray:
    """solver.ts:363-392: each load goes to the w DOF of the nearest node
    (the first node at the minimum distance), accumulated in float32."""
    F = np.zeros(mesh.nodeCount * DOFS_PER_NODE, np.float32)
    xy = mesh.nodes.reshape(-1, 2).astype(np.float64)
    for ld in loads:
        px, py = ld.position
        dist = np.sqrt((xy[:, 0] - px) ** 2 + (xy[:, 1] - py) ** 2)
        n = int(np.argmin(dist))
        F[n * DOFS_PER_NODE] = np.float32(np.float64(F[n * DOFS_PER_NODE]) + ld.magnitude)
    return F


def applyBCsToRHS(F: np.ndarray, constrainedDOFs) -> None:
    """solver.ts:400-407 (in place)."""
    for d in constrainedDOFs:
        F[int(d)] = 0.0


def element_areas(mesh: PlateMesh) -> np.ndarray:
    """Shoelace area of every element (float64 from the float32 nodes)."""
    npe = mesh.nodesPerElement
    xy = mesh.nodes.reshape(-1, 2).astype(np.float64)
    el = mesh.elements.astype(np.int64).reshape(-1, npe)
    x = xy[el, 0]
    y = xy[el, 1]
    s = np.sum(x * np.roll(y, -1, axis=1) - np.roll(x, -1, axis=1) * y, axis=1)
    return 0.5 * np.abs(s)


def pressure_load_vector(mesh: PlateMesh, pressure, out: Optional[np.ndarray] = None):
    """Nodal equivalent of a pressure (Pa, positive downward; scalar or one
    value per element): q_e * A_e / npe on the w DOF of each element node.
    Returned in float64 so that callers add point loads before the one
    final rounding to the float32 F of the solver interface."""
    npe = mesh.nodesPerElement
    F = np.zeros(mesh.nodeCount * DOFS_PER_NODE) if out is None else out
    q = np.broadcast_to(np.asarray(pressure, np.float64), (mesh.elementCount,))
    share = q * element_areas(mesh) / npe
    el = mesh.elements.astype(np.int64).reshape(-1, npe)
    np.add.at(F, el.reshape(-1) * DOFS_PER_NODE, np.repeat(share, npe))
    return F
