"""Element colouring (host side), mirroring src/lib/plate/coloring.ts.

Two elements conflict when they share a node; elements of one colour can be
applied in parallel with no scatter conflict.  The CUDA solver validates the
caller's colouring (recolouring greedily when two node-sharing elements
share a colour) and uses it in the colour-ordered K.x of pg_apply_k; the
persistent PCG kernel does not need it, because every (element, node)
task writes its own slot and each node sums its slots in a fixed order.
"""
from __future__ import annotations

import numpy as np

from .types import ElementColoring, PlateMesh


def _from_colors(element_colors: np.ndarray, count: int) -> ElementColoring:
    order = np.argsort(element_colors, kind="stable").astype(np.uint32)
    counts = np.bincount(element_colors, minlength=count)[:count]
    offs = np.concatenate([[0], np.cumsum(counts)])
    colors = [np.ascontiguousarray(order[offs[c]:offs[c + 1]], np.uint32) for c in range(count)]
    return ElementColoring(colors=colors, elementColors=element_colors.astype(np.uint8),
                           colorCount=count)


def computeElementColoring(mesh: PlateMesh) -> ElementColoring:
    """coloring.ts:38-81: colour = (i % 2) * 2 + (j % 2) on the element grid."""
    e = np.arange(mesh.elementCount, dtype=np.int64)
    i = e % mesh.gridNx
    j = e // mesh.gridNx
    return _from_colors(((i % 2) * 2 + (j % 2)).astype(np.int64), 4)


def _node_to_elements(mesh: PlateMesh):
    npe = mesh.nodesPerElement
    el = mesh.elements.astype(np.int64).reshape(-1, npe)
    owner = np.repeat(np.arange(mesh.elementCount, dtype=np.int64), npe)
    nodes = el.reshape(-1)
    order = np.argsort(nodes, kind="stable")
    ptr = np.zeros(mesh.nodeCount + 1, np.int64)
    np.add.at(ptr, nodes + 1, 1)
    ptr = np.cumsum(ptr)
    return ptr, owner[order], el


def computeElementColoringGreedy(mesh: PlateMesh) -> ElementColoring:
    """coloring.ts:92-177: first-fit over elements in index order; an
    element takes the smallest colour none of its node-sharing neighbours
    already has."""
    ptr, idx, el = _node_to_elements(mesh)
    ne = mesh.elementCount
    colors = np.full(ne, 255, np.int64)
    maxc = 0
    for e in range(ne):
        used = set()
        for n in el[e]:
            nb = idx[ptr[n]:ptr[n + 1]]
            cs = colors[nb]
            used.update(cs[(cs != 255) & (nb != e)].tolist())
        c = 0
        while c in used:
            c += 1
        colors[e] = c
        maxc = max(maxc, c)
    return _from_colors(colors, maxc + 1 if ne else 1)


def verifyColoring(mesh: PlateMesh, coloring: ElementColoring) -> bool:
    """coloring.ts:188-225: no two elements at a node share a colour."""
    ptr, idx, _el = _node_to_elements(mesh)
    ec = np.asarray(coloring.elementColors, np.int64)
    for n in range(mesh.nodeCount):
        cs = ec[idx[ptr[n]:ptr[n + 1]]]
        if cs.size != np.unique(cs).size:
            return False
    return True


def getColoringStats(coloring: ElementColoring) -> dict:
    """coloring.ts:235-253."""
    per = [len(c) for c in coloring.colors]
    lo, hi = min(per), max(per)
    return {"colorCount": coloring.colorCount, "elementsPerColor": per,
            "minElementsPerColor": lo, "maxElementsPerColor": hi,
            "balance": hi / lo if lo > 0 else float("inf")}
