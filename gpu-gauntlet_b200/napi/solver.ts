/**
 * CUDA (B200) drop-in for src/lib/plate/gpu/solver.ts of the reference.
 *
 * Same exports and signatures:
 *   solveGPU(mesh, material, coloring, F, constrainedDOFs, options)
 *     -> Promise<GPUSolveResult>                      (solver.ts:80-104)
 *   clearPipelineCache()                              (solver.ts:601-603)
 *   isWebGPUAvailable() -- kept under the reference name; true when the
 *     CUDA addon loaded and a B200 is visible          (context.ts:19)
 * Same defaults (tolerance 1e-6, maxIterations 1000) and result fields;
 * `solution` is a Float32Array of 3 * nodeCount values [w, thx, thy].
 *
 * Differences, on purpose: there is no CPU fallback -- forceCPU, a missing
 * addon or a missing device reject the promise (usedGPU is always true);
 * NaN/Inf in F rejects with PG_ENONFINITE; gpuTimeMs is the addon call's
 * wall time (set-up and solve, as the reference measures it).
 */
import type { ElementColoring, PlateMaterial, PlateMesh } from '../types';

export interface GPUSolverOptions {
  tolerance?: number;
  maxIterations?: number;
  forceCPU?: boolean;
  /** 'fp64' (default) or 'mixed' (FP32 inner iterations, FP64 residual checks) */
  precision?: 'fp64' | 'mixed';
  /** 'block-jacobi' (default, the reference's) or 'two-level' (plus a coarse correction) */
  preconditioner?: 'block-jacobi' | 'two-level';
  /** 'block-jacobi' (default) or 'chebyshev' (two Chebyshev steps for D^-1 K) */
  smoother?: 'block-jacobi' | 'chebyshev';
  /** 'reference' (default: ||r|| < tol or ||r||/||b|| < tol) or 'relative' (||r||/||b|| < tol) */
  stopRule?: 'reference' | 'relative';
  /** CUDA device index (default 0); each device gets its own solver context */
  device?: number;
}

export interface GPUSolveResult {
  solution: Float32Array;
  iterations: number;
  finalResidual: number;
  converged: boolean;
  gpuTimeMs: number;
  usedGPU: boolean;
}

interface AddonResult {
  solution: Float64Array;
  iterations: number;
  finalResidual: number;
  converged: boolean;
  gpuTimeMs: number;
}

interface Addon {
  solve(problem: Record<string, unknown>): Promise<AddonResult>;
  solveLoadCases(problem: Record<string, unknown>): Promise<AddonResult[]>;
  isAvailable(): boolean;
  clearCache(): void;
}

let addon: Addon | null = null;
let addonError: Error | null = null;

function loadAddon(): Addon {
  if (addon) return addon;
  if (addonError) throw addonError;
  try {
    // eslint-disable-next-line @typescript-eslint/no-var-requires
    addon = require('./plategpu_napi.node') as Addon;
    return addon;
  } catch (e) {
    addonError = new Error(`plategpu addon not loadable: ${(e as Error).message}`);
    throw addonError;
  }
}

export function isWebGPUAvailable(): boolean {
  try {
    return loadAddon().isAvailable();
  } catch {
    return false;
  }
}

export function clearPipelineCache(): void {
  try {
    loadAddon().clearCache();
  } catch {
    /* nothing cached without the addon */
  }
}

function addonProblem(
  mesh: PlateMesh,
  material: PlateMaterial,
  coloring: ElementColoring,
  F: Float32Array,
  constrainedDOFs: Set<number>,
  options: GPUSolverOptions
): Record<string, unknown> {
  if (options.forceCPU) {
    throw new Error('PG_EUNSUPPORTED: forceCPU requested; this solver has no CPU path');
  }
  const nodesPerElement = mesh.nodesPerElement ?? 4;
  const dofCount = mesh.nodeCount * 3;
  const constrained = new Uint8Array(dofCount);
  for (const dof of constrainedDOFs) constrained[dof] = 1;
  const colorOffsets = new Uint32Array(coloring.colorCount + 1);
  for (let c = 0; c < coloring.colorCount; c++) {
    colorOffsets[c + 1] = colorOffsets[c] + coloring.colors[c].length;
  }
  const elementsByColor = new Uint32Array(mesh.elementCount);
  for (let c = 0; c < coloring.colorCount; c++) {
    elementsByColor.set(coloring.colors[c], colorOffsets[c]);
  }
  return {
    nodeCount: mesh.nodeCount,
    elementCount: mesh.elementCount,
    nodesPerElement,
    nodes: mesh.nodes,
    elements: mesh.elements,
    colorOffsets,
    elementsByColor,
    E: material.E,
    nu: material.nu,
    t: material.t,
    F,
    constrained,
    tolerance: options.tolerance ?? 1e-6,
    maxIterations: options.maxIterations ?? 1000,
    precision: options.precision === 'mixed' ? 1 : 0,
    preconditioner: options.preconditioner === 'two-level' ? 1 : 0,
    smoother: options.smoother === 'chebyshev' ? 1 : 0,
    stopRule: options.stopRule === 'relative' ? 1 : 0,
    device: options.device ?? 0,
  };
}

function toResult(r: AddonResult): GPUSolveResult {
  return {
    solution: Float32Array.from(r.solution),
    iterations: r.iterations,
    finalResidual: r.finalResidual,
    converged: r.converged,
    gpuTimeMs: r.gpuTimeMs,
    usedGPU: true,
  };
}

export async function solveGPU(
  mesh: PlateMesh,
  material: PlateMaterial,
  coloring: ElementColoring,
  F: Float32Array,
  constrainedDOFs: Set<number>,
  options: GPUSolverOptions = {}
): Promise<GPUSolveResult> {
  const r = await loadAddon().solve(addonProblem(mesh, material, coloring, F, constrainedDOFs, options));
  return toResult(r);
}

/**
 * Several loads of one plate (the reference calls solveGPU once per load):
 * the loads run in lockstep on the GPU, up to four per persistent launch,
 * each with its own iterations and stop.  One result per load, in order;
 * gpuTimeMs is the wall clock of the whole call.
 */
export async function solveGPULoadCases(
  mesh: PlateMesh,
  material: PlateMaterial,
  coloring: ElementColoring,
  loads: Float32Array[],
  constrainedDOFs: Set<number>,
  options: GPUSolverOptions = {}
): Promise<GPUSolveResult[]> {
  const n = mesh.nodeCount * 3;
  const all = new Float32Array(n * loads.length);
  loads.forEach((f, k) => {
    if (f.length !== n) throw new Error(`PG_EINVAL: load ${k} has ${f.length} entries, expected ${n}`);
    all.set(f, k * n);
  });
  const problem = addonProblem(mesh, material, coloring, all, constrainedDOFs, options);
  problem.cases = loads.length;
  const t0 = Date.now();
  const rs = await loadAddon().solveLoadCases(problem);
  const ms = Date.now() - t0;
  return rs.map((r) => ({ ...toResult(r), gpuTimeMs: ms }));
}
