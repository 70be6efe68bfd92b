"""solveGPU with the reference GPU-solver interface, on the CUDA library.

Mirrors src/lib/plate/gpu/solver.ts:
  solveGPU(mesh, material, coloring, F, constrainedDOFs, options)  :80-104
  clearPipelineCache()                                            :601-603
  isWebGPUAvailable() (gpu/context.ts:19), here "is a B200 usable"
Same arguments, defaults (tolerance 1e-6, maxIterations 1000) and result
fields.  Deliberate differences: there is no CPU fallback -- forceCPU, a
missing library or a missing device raise PlateGPUError instead of quietly
solving on the CPU (usedGPU is therefore always True); NaN/Inf in F raise
PG_ENONFINITE.  solveGPUAsync returns an awaitable, as the TypeScript
function returns a Promise.  solveGPULoadCases solves several loads of one
plate together (the reference calls solveGPU once per load).
"""
from __future__ import annotations

import asyncio
import time
from typing import Dict, List, Optional

import numpy as np

from . import _lib
from .problem import constrained_mask
from .types import ElementColoring, GPUSolveResult, GPUSolverOptions, PlateMaterial, PlateMesh

_contexts: Dict[int, _lib.Context] = {}

_PREC = {"fp64": _lib.PG_PREC_FP64, "mixed": _lib.PG_PREC_MIXED}
_STOP = {"reference": _lib.PG_STOP_REFERENCE, "relative": _lib.PG_STOP_RELATIVE}
_PRECOND = {"block-jacobi": _lib.PG_PRECOND_BLOCK_JACOBI, "two-level": _lib.PG_PRECOND_TWO_LEVEL}
_SMOOTHER = {"block-jacobi": _lib.PG_SMOOTHER_BLOCK_JACOBI, "chebyshev": _lib.PG_SMOOTHER_CHEBYSHEV}


def get_context(device: int = 0) -> _lib.Context:
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = _lib.Context(device)
        _contexts[device] = ctx
    return ctx


def isWebGPUAvailable() -> bool:
    """True when the CUDA library loads and a B200 (sm_100) is visible."""
    try:
        return bool(_lib.load().pg_is_available())
    except (ImportError, OSError):
        return False


def clearPipelineCache() -> None:
    """Drops the cached partition plans and device buffers."""
    for ctx in _contexts.values():
        ctx.clear_cache()


def _mask(mesh: PlateMesh, constrainedDOFs) -> np.ndarray:
    n = 3 * mesh.nodeCount
    if isinstance(constrainedDOFs, np.ndarray) and constrainedDOFs.dtype == np.uint8 \
            and constrainedDOFs.size == n:
        return np.ascontiguousarray(constrainedDOFs)
    return constrained_mask(n, constrainedDOFs)


def _option(table, value, name):
    if value not in table:
        raise _lib.PlateGPUError(_lib.PG_EINVAL, f"unknown {name} {value!r}: one of {sorted(table)}")
    return table[value]


def _make_options(options: GPUSolverOptions) -> _lib.PgOptions:
    return _lib.make_options(
        tolerance=1e-6 if options.tolerance is None else options.tolerance,
        max_iterations=1000 if options.maxIterations is None else options.maxIterations,
        precision=_option(_PREC, options.precision, "precision"),
        stop_rule=_option(_STOP, options.stopRule, "stopRule"),
        preconditioner=_option(_PRECOND, options.preconditioner, "preconditioner"),
        smoother=_option(_SMOOTHER, options.smoother, "smoother"))


def solveGPU(mesh: PlateMesh, material: PlateMaterial, coloring: Optional[ElementColoring],
             F: np.ndarray, constrainedDOFs, options: Optional[GPUSolverOptions] = None,
             device: int = 0) -> GPUSolveResult:
    """Solves K x = F on the GPU; see the module docstring."""
    options = options or GPUSolverOptions()
    if options.forceCPU:
        raise _lib.PlateGPUError(_lib.PG_EUNSUPPORTED,
                                 "forceCPU requested: this solver has no CPU path")
    F = np.asarray(F)
    if F.size != 3 * mesh.nodeCount:
        raise _lib.PlateGPUError(_lib.PG_EINVAL,
                                 f"F has {F.size} entries, expected {3 * mesh.nodeCount}")
    opts = _make_options(options)
    ctx = get_context(device)
    prob = _lib.Problem(mesh, material, coloring, F, _mask(mesh, constrainedDOFs))
    x, info = ctx.solve(prob, opts)
    sol = x if options.returnFloat64 else x.astype(np.float32)
    return GPUSolveResult(solution=sol, iterations=int(info.iterations),
                          finalResidual=float(info.final_residual),
                          converged=bool(info.converged), gpuTimeMs=float(info.total_ms),
                          usedGPU=True, info=info.as_dict())


def solveGPULoadCases(mesh: PlateMesh, material: PlateMaterial, coloring: Optional[ElementColoring],
                      loads, constrainedDOFs, options: Optional[GPUSolverOptions] = None,
                      device: int = 0, casesPerLaunch: int = 0) -> List[GPUSolveResult]:
    """solveGPU for several loads of one plate (pg_solve_load_cases): one
    GPUSolveResult per load, in order.  The loads share the plate's set-up
    and run in lockstep, up to casesPerLaunch (0 = automatic) per persistent
    launch; gpuTimeMs is the wall clock of the whole call."""
    options = options or GPUSolverOptions()
    if options.forceCPU:
        raise _lib.PlateGPUError(_lib.PG_EUNSUPPORTED,
                                 "forceCPU requested: this solver has no CPU path")
    F = np.stack([np.asarray(f, np.float32).reshape(-1) for f in loads]) if len(loads) else None
    if F is None or F.shape[1] != 3 * mesh.nodeCount:
        raise _lib.PlateGPUError(_lib.PG_EINVAL, f"each load needs {3 * mesh.nodeCount} entries")
    opts = _make_options(options)
    ctx = get_context(device)
    prob = _lib.Problem(mesh, material, coloring, F[0], _mask(mesh, constrainedDOFs))
    t0 = time.perf_counter()
    X, infos = ctx.solve_load_cases(prob, F, opts, casesPerLaunch)
    ms = (time.perf_counter() - t0) * 1e3
    out = []
    for x, info in zip(X, infos):
        out.append(GPUSolveResult(solution=x if options.returnFloat64 else x.astype(np.float32),
                                  iterations=int(info.iterations), finalResidual=float(info.final_residual),
                                  converged=bool(info.converged), gpuTimeMs=ms, usedGPU=True,
                                  info=info.as_dict()))
    return out


async def solveGPUAsync(*args, **kwargs) -> GPUSolveResult:
    """Awaitable form of solveGPU (the reference returns a Promise)."""
    return await asyncio.to_thread(solveGPU, *args, **kwargs)
