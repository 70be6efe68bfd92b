"""Host helpers of bench.py (no GPU): the batch methods' options, the
options copy the load-case arm uses, and the seeded load cases."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from plategpu import _lib, workloads  # noqa: E402


def test_batch_methods_map_to_their_options():
    want = {"mixed_two_level": (_lib.PG_PREC_MIXED, _lib.PG_PRECOND_TWO_LEVEL, _lib.PG_SMOOTHER_BLOCK_JACOBI),
            "fp64_two_level": (_lib.PG_PREC_FP64, _lib.PG_PRECOND_TWO_LEVEL, _lib.PG_SMOOTHER_BLOCK_JACOBI),
            "fp64_two_level_cheb": (_lib.PG_PREC_FP64, _lib.PG_PRECOND_TWO_LEVEL, _lib.PG_SMOOTHER_CHEBYSHEV),
            "fp64_block_jacobi": (_lib.PG_PREC_FP64, _lib.PG_PRECOND_BLOCK_JACOBI, _lib.PG_SMOOTHER_BLOCK_JACOBI)}
    assert set(want) == set(bench.BATCH_METHODS)
    for name, (prec, pre, smo) in want.items():
        o = bench.batch_options(name)
        assert (o.precision, o.preconditioner, o.smoother) == (prec, pre, smo)
        assert o.tolerance == 2e-7 and o.stop_rule == _lib.PG_STOP_RELATIVE and o.fallback == 1


def test_options_copy_changes_only_what_it_is_asked_to():
    o = _lib.make_options(tolerance=5e-6, precision=_lib.PG_PREC_MIXED, smoother=_lib.PG_SMOOTHER_CHEBYSHEV,
                          reliable_delta=0.01)
    c = bench._lib_options_copy(o, tolerance=2e-6)
    assert c.tolerance == 2e-6 and o.tolerance == 5e-6
    for f, _t in type(o)._fields_:
        if f != "tolerance":
            assert getattr(c, f) == getattr(o, f), f


def test_case_loads_first_is_the_workload_load_and_constraints_hold():
    wl = workloads.plate_q4_32()
    F = bench.case_loads(wl, 4)
    assert F.shape == (4, wl.n_dof) and F.dtype == np.float32
    np.testing.assert_array_equal(F[0], wl.F)
    assert not F[:, wl.cons_mask != 0].any()
    assert len({f.tobytes() for f in F}) == 4
    np.testing.assert_array_equal(F, bench.case_loads(wl, 4))  # seeded


def test_every_other_config_has_tolerances_and_data():
    for name in ("plate_q4_32", "plate_dkt_200", "plate_holes_dkt", "plate_q4_141"):
        assert name in bench.TOLERANCES and name in bench.WORKLOAD_DATA
        assert name in workloads.WORKLOADS
