"""Plate solver data types, mirroring the reference TypeScript interfaces.

Each class follows one interface of cseifert512/gpu-gauntlet:
  PlateMaterial, PlateSupport, PlateLoad, PlateMesh, ElementColoring
      src/lib/plate/types.ts:14-102
  GPUSolverOptions, GPUSolveResult
      src/lib/plate/gpu/solver.ts:35-60
Array fields keep the reference element types (Float32Array -> float32,
Uint32Array -> uint32, Uint8Array -> uint8).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

DOFS_PER_NODE = 3  # types.ts:176
NODES_PER_ELEMENT = 4  # types.ts:179
DOFS_PER_ELEMENT = 12  # types.ts:182
NODES_PER_TRIANGLE = 3  # types.ts:185
DOFS_PER_TRIANGLE = 9  # types.ts:188


def computeFlexuralRigidity(mat: "PlateMaterial") -> float:
    """D = E t^3 / (12 (1 - nu^2))  (types.ts:26-28)."""
    return (mat.E * mat.t ** 3) / (12 * (1 - mat.nu ** 2))


@dataclass
class PlateMaterial:
    """types.ts:14-21.  ``elem_t`` is an extension: an optional per-element
    thickness (float32, one per element) that overrides ``t``."""

    E: float
    nu: float
    t: float
    elem_t: Optional[np.ndarray] = None


@dataclass
class PlateSupport:
    """types.ts:47-51: type is 'pinned' | 'fixed' | 'roller'; location is a
    node index or 'all_edges'."""

    type: str
    location: Union[int, str]


@dataclass
class PlateLoad:
    """types.ts:57-62: point load in N at (x, y) m, positive downward."""

    position: Tuple[float, float]
    magnitude: float


@dataclass
class PlateMesh:
    """types.ts:73-89."""

    nodes: np.ndarray  # float32 [x0, y0, x1, y1, ...]
    elements: np.ndarray  # uint32, nodesPerElement per element
    boundaryNodes: np.ndarray  # uint32
    nodeCount: int
    elementCount: int
    nodesPerElement: int = 4
    gridNx: int = 0
    gridNy: int = 0

    def __post_init__(self):
        self.nodes = np.ascontiguousarray(self.nodes, dtype=np.float32)
        self.elements = np.ascontiguousarray(self.elements, dtype=np.uint32)
        self.boundaryNodes = np.ascontiguousarray(self.boundaryNodes, dtype=np.uint32)


@dataclass
class ElementColoring:
    """types.ts:95-102: per-colour element lists, the colour of each
    element, and the number of colours."""

    colors: List[np.ndarray]
    elementColors: np.ndarray
    colorCount: int

    def flat(self) -> Tuple[np.ndarray, np.ndarray]:
        """(color_offsets int32[colorCount+1], elements_by_color uint32[Ne]) --
        the layout of the reference's elementsByColor buffer
        (gpu/buffers.ts:143-170, gpu/solver.ts:143-150)."""
        counts = [len(c) for c in self.colors]
        offsets = np.zeros(len(counts) + 1, np.int32)
        offsets[1:] = np.cumsum(counts)
        flat = (np.concatenate([np.asarray(c, np.uint32) for c in self.colors])
                if counts else np.zeros(0, np.uint32))
        return offsets, np.ascontiguousarray(flat, np.uint32)


@dataclass
class GPUSolverOptions:
    """gpu/solver.ts:35-42 plus B200 extensions.

    tolerance / maxIterations / forceCPU keep the reference meaning (defaults
    1e-6 and 1000 as in gpu/solver.ts:121-122).  forceCPU is rejected: this
    solver has no CPU path.  Extensions: ``precision`` ('fp64' plain FP64
    PCG, 'mixed' FP32 inner iterations with FP64 residual replacement) and
    ``stopRule`` ('reference': ||r|| < tol or ||r||/||b|| < tol on the
    recursive residual, gpu/solver.ts:516; 'relative': ||r||/||b|| < tol),
    ``preconditioner`` ('block-jacobi', the reference's; 'two-level': plus a
    coarse correction with the plate's rigid modes on one aggregate per
    thread block) and ``smoother`` ('block-jacobi'; 'chebyshev': two
    Chebyshev steps for D^-1 K in place of D^-1)."""

    tolerance: Optional[float] = None
    maxIterations: Optional[int] = None
    forceCPU: bool = False
    precision: str = "fp64"
    stopRule: str = "reference"
    preconditioner: str = "block-jacobi"
    smoother: str = "block-jacobi"
    returnFloat64: bool = False


@dataclass
class GPUSolveResult:
    """gpu/solver.ts:47-60.  ``solution`` is float32 [w0, tx0, ty0, ...]
    (float64 when GPUSolverOptions.returnFloat64); usedGPU is always True.
    ``info`` carries the extended per-solve statistics."""

    solution: np.ndarray
    iterations: int
    finalResidual: float
    converged: bool
    gpuTimeMs: float
    usedGPU: bool = True
    info: dict = field(default_factory=dict)
