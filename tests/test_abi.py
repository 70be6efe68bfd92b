"""The C ABI library: loads without a GPU, exports every declared symbol,
struct layouts agree with the header, host-only hooks work."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from plategpu import _lib, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "plategpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pg_[a-z_]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    L = _lib.load()
    names = declared_functions()
    assert len(names) >= 13
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTED)


def test_struct_layout_matches_header():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "plategpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(pg_problem), sizeof(pg_options), sizeof(pg_info),
         offsetof(pg_problem, F), offsetof(pg_options, phase_timing), offsetof(pg_info, plan_cached),
         offsetof(pg_info, phase_us));
  return 0;
}
"""
    import ctypes as C
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True,
                                               check=True).stdout.split()]
    assert vals == [C.sizeof(_lib.PgProblem), C.sizeof(_lib.PgOptions), C.sizeof(_lib.PgInfo),
                    _lib.PgProblem.F.offset, _lib.PgOptions.phase_timing.offset,
                    _lib.PgInfo.plan_cached.offset, _lib.PgInfo.phase_us.offset]


def test_defaults_match_reference():
    import ctypes as C
    o = _lib.PgOptions()
    _lib.load().pg_options_default(C.byref(o))
    assert o.tolerance == 1e-6 and o.max_iterations == 1000  # gpu/solver.ts:121-122
    assert o.struct_size == C.sizeof(_lib.PgOptions)


def test_null_arguments_rejected():
    import ctypes as C
    L = _lib.load()
    assert L.pg_solve(None, None, None, None, None) == _lib.PG_EINVAL
    assert L.pg_create(0, None) == _lib.PG_EINVAL


@pytest.mark.skipif(_lib.load().pg_is_available() == 1, reason="a B200 is present")
def test_no_device_fails_loudly():
    import ctypes as C
    L = _lib.load()
    h = C.c_void_p()
    st = L.pg_create(0, C.byref(h))
    assert st in (_lib.PG_ECUDA, _lib.PG_EINVAL)
    assert len(L.pg_last_error(None)) > 0
    from plategpu import solveGPU, isWebGPUAvailable, PlateGPUError
    assert not isWebGPUAvailable()
    wl = workloads.plate_q4(8, 0)
    with pytest.raises(PlateGPUError):
        solveGPU(wl.mesh, wl.material, wl.coloring, wl.F, wl.constrainedDOFs)


@pytest.mark.parametrize("name", ["plate_q4_32", "plate_q4_141"])
@pytest.mark.parametrize("ctas", [1, 7, 64, 148])
def test_plan_invariants(name, ctas):
    wl = workloads.WORKLOADS[name]()
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    st = _lib.plan_inspect(pr, ctas)
    assert st["violations"] == 0
    assert st["parts"] == min(ctas, wl.mesh.nodeCount)
    assert st["recolored"] == 0 and st["colors"] == 4


def test_plan_recolors_conflicting_coloring():
    from plategpu.types import ElementColoring
    wl = workloads.plate_q4(10, 0)
    one = ElementColoring(colors=[np.arange(100, dtype=np.uint32)],
                          elementColors=np.zeros(100, np.uint8), colorCount=1)
    pr = _lib.Problem(wl.mesh, wl.material, one, wl.F, wl.cons_mask)
    st = _lib.plan_inspect(pr, 5)
    assert st["recolored"] == 1 and st["violations"] == 0 and st["colors"] >= 4


def test_plan_rejects_bad_inputs():
    wl = workloads.plate_q4(6, 0)
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    pr.elements[3] = 10_000  # node index out of range
    with pytest.raises(_lib.PlateGPUError, match="out of range"):
        _lib.plan_inspect(pr, 2)
    pr2 = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    pr2.elements_by_color[0] = pr2.elements_by_color[1]  # an element listed twice
    with pytest.raises(_lib.PlateGPUError, match="once"):
        _lib.plan_inspect(pr2, 2)


def test_dkt_plan_invariants():
    from plategpu import coloring, mesher
    from plategpu.types import PlateMaterial
    m = mesher.split_triangle_mesh(10, 10, 30, 30, jitter=0.2, seed=2)
    c = coloring.computeElementColoringGreedy(m)
    pr = _lib.Problem(m, PlateMaterial(2.1e11, 0.3, 0.1), c)
    st = _lib.plan_inspect(pr, 37)
    assert st["violations"] == 0 and st["parts"] == 37


@pytest.mark.parametrize("ctas", [1, 7, 148])
def test_plan_invariants_two_ring_halo(ctas):
    wl = workloads.plate_q4_141()
    pr = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
    one = _lib.plan_inspect(pr, ctas, rings=1)
    two = _lib.plan_inspect(pr, ctas, rings=2)
    assert two["violations"] == 0 and two["parts"] == one["parts"]
    if ctas > 1:  # ring-1 nodes carry tasks and a second ghost layer appears
        assert two["max_part_tasks"] > one["max_part_tasks"]
        assert two["ghost_nodes"] > one["ghost_nodes"]
        assert two["max_local_nodes"] > one["max_local_nodes"]
    else:
        assert two == one


def test_dkt_plan_invariants_two_ring_halo():
    from plategpu import coloring, mesher
    from plategpu.types import PlateMaterial
    m = mesher.split_triangle_mesh(10, 10, 30, 30, jitter=0.2, seed=2)
    c = coloring.computeElementColoringGreedy(m)
    pr = _lib.Problem(m, PlateMaterial(2.1e11, 0.3, 0.1), c)
    assert _lib.plan_inspect(pr, 37, rings=2)["violations"] == 0
    with pytest.raises(_lib.PlateGPUError, match="rings"):
        _lib.plan_inspect(pr, 37, rings=3)


def test_learned_struct_layouts_match_header():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "plategpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(pg_train_options), offsetof(pg_train_options, seed),
         sizeof(pg_train_info), offsetof(pg_train_info, epoch_val_loss), sizeof(pg_learned_stats),
         offsetof(pg_learned_stats, replacements));
  return 0;
}
"""
    import ctypes as C
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True,
                                               check=True).stdout.split()]
    assert vals == [C.sizeof(_lib.PgTrainOptions), _lib.PgTrainOptions.seed.offset,
                    C.sizeof(_lib.PgTrainInfo), _lib.PgTrainInfo.epoch_val_loss.offset,
                    C.sizeof(_lib.PgLearnedStats), _lib.PgLearnedStats.replacements.offset]


def test_train_options_defaults():
    import ctypes as C
    o = _lib.PgTrainOptions()
    _lib.load().pg_train_options_default(C.byref(o))
    assert o.struct_size == C.sizeof(_lib.PgTrainOptions)
    assert o.epochs == 20 and o.batch == 32 and abs(o.lr - 1e-3) < 1e-9 and o.cosine == 1


def test_batch_info_layout_matches_header():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "plategpu.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(pg_batch_info), offsetof(pg_batch_info, graph), sizeof(pg_info),
         offsetof(pg_info, global_path));
  return 0;
}
"""
    import ctypes as C
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True,
                                               check=True).stdout.split()]
    assert vals == [C.sizeof(_lib.PgBatchInfo), _lib.PgBatchInfo.graph.offset, C.sizeof(_lib.PgInfo),
                    _lib.PgInfo.global_path.offset]
