"""The Node-API addon builds against the C ABI and exports the module entry.

Node is not installed in this image (nor on the GPU box), so the addon
cannot be loaded here; this checks that it compiles, that Node would find
its entry point, and that every function it needs from Node is a stable
Node-API symbol it leaves for the node binary to supply.
"""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NAPI = os.path.join(ROOT, "gpu-gauntlet_b200", "napi")


def test_addon_builds_and_exports_entry():
    subprocess.run(["make", "-s", "-C", NAPI, "plategpu_napi.node"], check=True)
    out = subprocess.run(["nm", "-D", os.path.join(NAPI, "plategpu_napi.node")],
                         capture_output=True, text=True, check=True).stdout
    defined = {l.split()[-1] for l in out.splitlines() if " T " in l}
    undefined = {l.split()[-1] for l in out.splitlines() if l.strip().startswith("U ")}
    assert "napi_register_module_v1" in defined
    needed = {u for u in undefined if u.startswith("napi_")}
    assert {"napi_create_promise", "napi_create_async_work", "napi_queue_async_work",
            "napi_resolve_deferred", "napi_reject_deferred"} <= needed
    assert {"pg_solve", "pg_solve_load_cases", "pg_create", "pg_last_error"} <= undefined


def test_typescript_wrapper_keeps_reference_signature():
    src = open(os.path.join(NAPI, "solver.ts")).read()
    assert ("export async function solveGPU(\n  mesh: PlateMesh,\n  material: PlateMaterial,\n"
            "  coloring: ElementColoring,\n  F: Float32Array,\n  constrainedDOFs: Set<number>,\n"
            "  options: GPUSolverOptions = {}\n): Promise<GPUSolveResult>") in src
    for name in ("isWebGPUAvailable", "clearPipelineCache"):
        assert f"export function {name}(" in src
    assert "export async function solveGPULoadCases(" in src
