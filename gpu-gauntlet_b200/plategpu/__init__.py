"""plategpu: B200-native matrix-free plate-bending PCG solver.

Host side of the solver: the reference GPU-solver interface (solveGPU and
friends), the problem-definition helpers upstream of it (mesher, colouring,
supports, loads) and the seeded workloads.  The solve itself runs in the
CUDA library libplategpu.so through the C ABI of include/plategpu.h.
"""
from .types import (DOFS_PER_ELEMENT, DOFS_PER_NODE, DOFS_PER_TRIANGLE, NODES_PER_ELEMENT,
                    NODES_PER_TRIANGLE, ElementColoring, GPUSolveResult, GPUSolverOptions,
                    PlateLoad, PlateMaterial, PlateMesh, PlateSupport, computeFlexuralRigidity)
from .mesher import generateRectangularMesh, getElementCoords, split_triangle_mesh
from .coloring import (computeElementColoring, computeElementColoringGreedy, getColoringStats,
                       verifyColoring)
from .problem import (applyBCsToRHS, buildLoadVector, constrained_mask, identifyConstrainedDOFs,
                      pressure_load_vector)
from .solver import (clearPipelineCache, isWebGPUAvailable, solveGPU, solveGPUAsync,
                     solveGPULoadCases)
from .postprocess import (computeMoments, extractVerticalDisplacements, findMaxDisplacement,
                          findMaxMoments)
from ._lib import PlateGPUError
