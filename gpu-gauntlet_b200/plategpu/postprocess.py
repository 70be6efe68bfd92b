"""Post-processing of a solution, with the reference's interface.

Mirrors src/lib/plate/postprocess.ts:
  computeMoments(mesh, displacements, material)   :40-264  (GPU, pg_moments)
  extractVerticalDisplacements(displacements, n)  :272-281
  findMaxDisplacement(w, nodes)                   :290-318
  findMaxMoments(Mx, My, Mxy)                     :323-343
computeMoments returns float32 arrays like the reference's Float32Arrays
(the device computes in FP64 and rounds once).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .types import PlateMaterial, PlateMesh


def computeMoments(mesh: PlateMesh, displacements, material: PlateMaterial, device: int = 0):
    """Nodal bending moments {Mx, My, Mxy} of a displacement vector."""
    from .solver import get_context
    prob = _lib.Problem(mesh, material, None)
    Mx, My, Mxy = get_context(device).moments(prob, np.asarray(displacements, np.float64))
    return {"Mx": Mx.astype(np.float32), "My": My.astype(np.float32), "Mxy": Mxy.astype(np.float32)}


def extractVerticalDisplacements(displacements, nodeCount: int) -> np.ndarray:
    """w of every node from [w0, thx0, thy0, w1, ...]."""
    return np.asarray(displacements, np.float32)[0: 3 * nodeCount: 3].copy()


def findMaxDisplacement(w, nodes) -> dict:
    """Largest |w| (first such node), returned with its sign and position."""
    w = np.asarray(w, np.float32)
    i = int(np.argmax(np.abs(w))) if w.size else 0
    xy = np.asarray(nodes, np.float32)
    return {"maxW": float(w[i]) if w.size else float("-inf"), "nodeIndex": i,
            "x": float(xy[2 * i]) if xy.size else float("nan"),
            "y": float(xy[2 * i + 1]) if xy.size else float("nan")}


def findMaxMoments(Mx, My, Mxy) -> dict:
    """Signed value of largest magnitude of each moment (first on ties).

    Deliberate difference: the reference starts each maximum at -Infinity
    and compares magnitudes, and since |-Infinity| exceeds every value it
    returns -Infinity for every input; this returns the intended value."""
    def big(a):
        a = np.asarray(a, np.float32)
        return float(a[int(np.argmax(np.abs(a)))]) if a.size else float("-inf")
    return {"maxMx": big(Mx), "maxMy": big(My), "maxMxy": big(Mxy)}
