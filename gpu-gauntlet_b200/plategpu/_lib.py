"""ctypes binding of libplategpu.so (the C ABI declared in include/plategpu.h).

The library is built in-tree by ``plategpu.build.build_library()`` (nvcc,
sm_100a).  Loading fails loudly when it is missing: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libplategpu.so")

PG_OK, PG_EINVAL, PG_ENOMEM, PG_ECUDA, PG_ETIMEOUT, PG_ENONFINITE, PG_EUNSUPPORTED = range(7)
STATUS_NAMES = {0: "PG_OK", 1: "PG_EINVAL", 2: "PG_ENOMEM", 3: "PG_ECUDA", 4: "PG_ETIMEOUT",
                5: "PG_ENONFINITE", 6: "PG_EUNSUPPORTED"}
PG_PREC_FP64, PG_PREC_MIXED = 0, 1
PG_STOP_REFERENCE, PG_STOP_RELATIVE = 0, 1
PG_PRECOND_BLOCK_JACOBI, PG_PRECOND_TWO_LEVEL = 0, 1
PG_SMOOTHER_BLOCK_JACOBI, PG_SMOOTHER_CHEBYSHEV = 0, 1
(PG_STOP_CONVERGED, PG_STOP_MAX_ITER, PG_STOP_BREAKDOWN, PG_STOP_ZERO_RHS,
 PG_STOP_STAGNATED) = range(5)  # pg_stop_reason
STOP_REASONS = {0: "converged", 1: "max_iterations", 2: "breakdown", 3: "zero_rhs",
                4: "stagnated"}

# every symbol include/plategpu.h declares
EXPORTED = ("pg_options_default", "pg_is_available", "pg_create", "pg_destroy", "pg_last_error",
            "pg_clear_cache", "pg_set_stream", "pg_solve", "pg_plan_create", "pg_plan_solve_device",
            "pg_plan_destroy", "pg_apply_k", "pg_apply_k_static",
            "pg_block_jacobi", "pg_element_stiffness", "pg_plan_inspect",
            "pg_plan_inspect_halo", "pg_batch_create", "pg_batch_solve", "pg_batch_destroy",
            "pg_solve_batch", "pg_batch_schedule", "pg_partition_nodes", "pg_moments", "pg_plan_moments_device", "pg_solve_load_cases",
            "pg_net_create", "pg_net_destroy", "pg_net_param_count", "pg_net_set_params",
            "pg_net_get_params", "pg_net_forward", "pg_net_backward", "pg_net_adam_step",
            "pg_learned_create", "pg_learned_destroy", "pg_learned_make_pairs",
            "pg_train_options_default", "pg_learned_train", "pg_learned_loss",
            "pg_learned_solve_device", "pg_learned_solve", "pg_learned_apply_k")

PG_TRAIN_MAX_EPOCHS = 256
# pg_learned_solve modes
LEARNED_BLOCK_JACOBI, LEARNED_NETWORK, LEARNED_SMOOTHING_ONLY = 0, 1, 2


class PgProblem(C.Structure):
    _fields_ = [
        ("node_count", C.c_uint32),
        ("element_count", C.c_uint32),
        ("nodes_per_element", C.c_uint32),
        ("nodes", C.c_void_p),
        ("elements", C.c_void_p),
        ("color_count", C.c_uint32),
        ("color_offsets", C.c_void_p),
        ("elements_by_color", C.c_void_p),
        ("E", C.c_double),
        ("nu", C.c_double),
        ("t", C.c_double),
        ("elem_t", C.c_void_p),
        ("F", C.c_void_p),
        ("constrained", C.c_void_p),
    ]


class PgOptions(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("tolerance", C.c_double),
        ("max_iterations", C.c_int32),
        ("precision", C.c_int32),
        ("stop_rule", C.c_int32),
        ("ctas", C.c_int32),
        ("threads", C.c_int32),
        ("wait_timeout_ms", C.c_double),
        ("reliable_interval", C.c_int32),
        ("reliable_delta", C.c_double),
        ("phase_timing", C.c_int32),
        ("test_stall", C.c_int32),
        ("preconditioner", C.c_int32),
        ("trace_iteration", C.c_int32),
        ("smoother", C.c_int32),
        ("fallback", C.c_int32),
        ("batch_part_nodes", C.c_int32),
    ]


class PgBatchInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("count", C.c_int32),
        ("teams", C.c_int32),
        ("grid", C.c_int32),
        ("converged", C.c_int32),
        ("shared_bytes", C.c_int32),
        ("phases", C.c_int32),
        ("fallbacks", C.c_int32),
        ("setup_ms", C.c_double),
        ("solve_ms", C.c_double),
        ("total_ms", C.c_double),
        ("plate_ms_p50", C.c_double),
        ("plate_ms_p99", C.c_double),
        ("plate_ms_max", C.c_double),
        ("solves_per_s", C.c_double),
        ("graph", C.c_int32),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["status"] = STATUS_NAMES.get(d["status"], d["status"])
        return d


class PgInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("stop_reason", C.c_int32),
        ("final_residual", C.c_double),
        ("true_rel_residual", C.c_double),
        ("b_norm", C.c_double),
        ("setup_ms", C.c_double),
        ("solve_ms", C.c_double),
        ("total_ms", C.c_double),
        ("ctas", C.c_int32),
        ("threads", C.c_int32),
        ("reliable_updates", C.c_int32),
        ("plan_cached", C.c_int32),
        ("reductions", C.c_int32),
        ("shared_bytes", C.c_int32),
        ("coarse_dim", C.c_int32),
        ("fallback", C.c_int32),
        ("phase_us", C.c_double * 8),
        ("trace_ns", C.c_double * 6),
        ("smoother_lambda_max", C.c_double),
        ("global_path", C.c_int32),
        ("reserved", C.c_int32),
        ("plan_ms", C.c_double),
        ("coarse_ms", C.c_double),
        ("eigen_ms", C.c_double),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["phase_us"] = list(self.phase_us)
        d["trace_ns"] = list(self.trace_ns)
        d["stop_reason"] = STOP_REASONS.get(d["stop_reason"], d["stop_reason"])
        return d


class PgTrainOptions(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("epochs", C.c_int32),
        ("batch", C.c_int32),
        ("lr", C.c_float),
        ("cosine", C.c_int32),
        ("seed", C.c_uint64),
        ("val_count", C.c_int32),
        ("set_scales", C.c_int32),
        ("loss", C.c_int32),
    ]


class PgTrainInfo(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("batch", C.c_int32),
        ("loss_first_step", C.c_double),
        ("loss_last_step", C.c_double),
        ("val_loss_before", C.c_double),
        ("val_loss", C.c_double),
        ("train_ms", C.c_double),
        ("total_ms", C.c_double),
        ("epoch_loss", C.c_double * PG_TRAIN_MAX_EPOCHS),
        ("epoch_val_loss", C.c_double * PG_TRAIN_MAX_EPOCHS),
    ]


class PgLearnedStats(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("network_iterations", C.c_int32),
        ("network_off_at", C.c_int32),
        ("replacements", C.c_int32),
        ("pdl", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PlateGPUError(RuntimeError):
    """A non-OK pg_status; ``status`` holds the code name."""

    def __init__(self, status: int, message: str):
        self.status = STATUS_NAMES.get(status, str(status))
        self.code = status
        super().__init__(f"{self.status}: {message}")


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run plategpu.build.build_library() "
                          "(nvcc, sm_100a). There is no CPU fallback.")
    L = C.CDLL(LIB_PATH)
    P, I = C.c_void_p, C.c_int
    L.pg_options_default.argtypes = [C.POINTER(PgOptions)]
    L.pg_options_default.restype = None
    L.pg_is_available.argtypes = []
    L.pg_is_available.restype = I
    L.pg_create.argtypes = [I, C.POINTER(P)]
    L.pg_create.restype = I
    L.pg_destroy.argtypes = [P]
    L.pg_destroy.restype = None
    L.pg_last_error.argtypes = [P]
    L.pg_last_error.restype = C.c_char_p
    L.pg_clear_cache.argtypes = [P]
    L.pg_clear_cache.restype = I
    L.pg_set_stream.argtypes = [P, P]
    L.pg_set_stream.restype = I
    L.pg_solve.argtypes = [P, C.POINTER(PgProblem), C.POINTER(PgOptions), P, C.POINTER(PgInfo)]
    L.pg_solve.restype = I
    L.pg_solve_load_cases.argtypes = [P, C.POINTER(PgProblem), I, P, C.POINTER(PgOptions), I, P, P]
    L.pg_solve_load_cases.restype = I
    L.pg_plan_create.argtypes = [P, C.POINTER(PgProblem), C.POINTER(PgOptions), C.POINTER(P)]
    L.pg_plan_create.restype = I
    L.pg_plan_solve_device.argtypes = [P, C.POINTER(PgOptions), P, P, C.POINTER(PgInfo)]
    L.pg_plan_solve_device.restype = I
    L.pg_plan_destroy.argtypes = [P]
    L.pg_plan_destroy.restype = None
    L.pg_apply_k.argtypes = [P, C.POINTER(PgProblem), P, P]
    L.pg_apply_k.restype = I
    L.pg_block_jacobi.argtypes = [P, C.POINTER(PgProblem), P]
    L.pg_block_jacobi.restype = I
    L.pg_element_stiffness.argtypes = [P, C.POINTER(PgProblem), P]
    L.pg_element_stiffness.restype = I
    L.pg_apply_k_static.argtypes = [C.POINTER(PgProblem), P, P, P, C.c_char_p, C.c_size_t]
    L.pg_apply_k_static.restype = I
    L.pg_plan_inspect.argtypes = [C.POINTER(PgProblem), I, P, C.c_char_p, C.c_size_t]
    L.pg_plan_inspect.restype = I
    L.pg_plan_inspect_halo.argtypes = [C.POINTER(PgProblem), I, I, P, C.c_char_p, C.c_size_t]
    L.pg_plan_inspect_halo.restype = I
    L.pg_batch_create.argtypes = [P, C.POINTER(PgProblem), I, C.POINTER(PgOptions), C.POINTER(P)]
    L.pg_batch_create.restype = I
    L.pg_batch_solve.argtypes = [P, C.POINTER(PgOptions), P, P, P, C.POINTER(PgBatchInfo)]
    L.pg_batch_solve.restype = I
    L.pg_batch_destroy.argtypes = [P]
    L.pg_batch_destroy.restype = None
    L.pg_solve_batch.argtypes = [P, C.POINTER(PgProblem), I, C.POINTER(PgOptions), P, P,
                                 C.POINTER(PgBatchInfo)]
    L.pg_solve_batch.restype = I
    L.pg_batch_schedule.argtypes = [P, I, I, I, P, P, P, P, P]
    L.pg_batch_schedule.restype = I
    L.pg_partition_nodes.argtypes = [P, C.c_uint32, I, P]
    L.pg_partition_nodes.restype = I
    L.pg_moments.argtypes = [P, C.POINTER(PgProblem), P, P, P, P]
    L.pg_moments.restype = I
    L.pg_plan_moments_device.argtypes = [P, P, P]
    L.pg_plan_moments_device.restype = I
    L.pg_net_create.argtypes = [P, I, I, C.c_uint64, C.POINTER(P)]
    L.pg_net_create.restype = I
    L.pg_net_destroy.argtypes = [P]
    L.pg_net_destroy.restype = None
    L.pg_net_param_count.argtypes = [P]
    L.pg_net_param_count.restype = C.c_int64
    L.pg_net_set_params.argtypes = [P, P, P]
    L.pg_net_set_params.restype = I
    L.pg_net_get_params.argtypes = [P, P, P]
    L.pg_net_get_params.restype = I
    L.pg_net_forward.argtypes = [P, I, P, P]
    L.pg_net_forward.restype = I
    L.pg_net_backward.argtypes = [P, I, P, P, P]
    L.pg_net_backward.restype = I
    L.pg_net_adam_step.argtypes = [P, P, C.c_float]
    L.pg_net_adam_step.restype = I
    L.pg_learned_create.argtypes = [P, P, P, C.POINTER(P)]
    L.pg_learned_create.restype = I
    L.pg_learned_destroy.argtypes = [P]
    L.pg_learned_destroy.restype = None
    L.pg_learned_make_pairs.argtypes = [P, I, P, P, P, P, P]
    L.pg_learned_make_pairs.restype = I
    L.pg_train_options_default.argtypes = [C.POINTER(PgTrainOptions)]
    L.pg_train_options_default.restype = None
    L.pg_learned_train.argtypes = [P, I, P, P, C.POINTER(PgTrainOptions), C.POINTER(PgTrainInfo)]
    L.pg_learned_train.restype = I
    L.pg_learned_loss.argtypes = [P, I, P, P, P]
    L.pg_learned_loss.restype = I
    L.pg_learned_solve_device.argtypes = [P, C.POINTER(PgOptions), I, P, P, C.POINTER(PgInfo),
                                          C.POINTER(PgLearnedStats)]
    L.pg_learned_solve_device.restype = I
    L.pg_learned_solve.argtypes = [P, C.POINTER(PgOptions), I, P, P, C.POINTER(PgInfo),
                                   C.POINTER(PgLearnedStats)]
    L.pg_learned_solve.restype = I
    L.pg_learned_apply_k.argtypes = [P, P, P]
    L.pg_learned_apply_k.restype = I
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


class Problem:
    """Owns contiguous copies of the arrays a PgProblem points at."""

    def __init__(self, mesh, material, coloring, F=None, constrained=None):
        self.nodes = np.array(mesh.nodes, np.float32, order="C")
        self.elements = np.array(mesh.elements, np.uint32, order="C")
        if coloring is not None:
            offs, flat = coloring.flat()
            self.color_offsets = np.array(offs, np.uint32, order="C")
            self.elements_by_color = np.array(flat, np.uint32, order="C")
            ncol = int(coloring.colorCount)
        else:
            self.color_offsets = self.elements_by_color = None
            ncol = 0
        self.elem_t = (None if getattr(material, "elem_t", None) is None
                       else np.array(material.elem_t, np.float32, order="C"))
        n = 3 * int(mesh.nodeCount)
        self.F = np.zeros(n, np.float32) if F is None else np.array(F, np.float32, order="C")
        if self.F.size != n:
            raise ValueError(f"F has {self.F.size} entries, expected {n}")
        self.cons = (np.zeros(n, np.uint8) if constrained is None
                     else np.array(constrained, np.uint8, order="C"))
        if self.cons.size != n:
            raise ValueError(f"constrained mask has {self.cons.size} entries, expected {n}")
        s = PgProblem()
        s.node_count = int(mesh.nodeCount)
        s.element_count = int(mesh.elementCount)
        s.nodes_per_element = int(mesh.nodesPerElement)
        s.nodes = _ptr(self.nodes)
        s.elements = _ptr(self.elements)
        s.color_count = ncol
        s.color_offsets = _ptr(self.color_offsets)
        s.elements_by_color = _ptr(self.elements_by_color)
        s.E, s.nu, s.t = float(material.E), float(material.nu), float(material.t)
        s.elem_t = _ptr(self.elem_t)
        s.F = _ptr(self.F)
        s.constrained = _ptr(self.cons)
        self.struct = s

    def set_F(self, F):
        F = np.ascontiguousarray(F, np.float32)
        if F.size != self.F.size:
            raise ValueError("F size mismatch")
        self.F = F
        self.struct.F = _ptr(F)


PLAN_STATS = ("parts", "colors", "recolored", "max_local_nodes", "max_owned_nodes",
              "max_part_tasks", "ghost_nodes", "violations")


def plan_inspect(prob: "Problem", ctas: int, rings: int = 1) -> dict:
    """pg_plan_inspect(_halo): host-only partition statistics and invariant check."""
    stats = np.zeros(8, np.int32)
    msg = C.create_string_buffer(256)
    st = load().pg_plan_inspect_halo(C.byref(prob.struct), int(ctas), int(rings), _ptr(stats),
                                     msg, 256)
    if st != PG_OK:
        raise PlateGPUError(st, msg.value.decode())
    return dict(zip(PLAN_STATS, stats.tolist()))


def make_options(tolerance=1e-6, max_iterations=1000, precision=PG_PREC_FP64,
                 stop_rule=PG_STOP_REFERENCE, ctas=0, threads=0, wait_timeout_ms=None,
                 reliable_interval=0, reliable_delta=0.0, phase_timing=False,
                 test_stall=False, preconditioner=PG_PRECOND_BLOCK_JACOBI,
                 trace_iteration=0, smoother=PG_SMOOTHER_BLOCK_JACOBI,
                 fallback=True, batch_part_nodes=0) -> PgOptions:
    o = PgOptions()
    load().pg_options_default(C.byref(o))
    o.tolerance = float(tolerance)
    o.max_iterations = int(max_iterations)
    o.precision = int(precision)
    o.stop_rule = int(stop_rule)
    o.ctas = int(ctas)
    o.threads = int(threads)
    if wait_timeout_ms is not None:
        o.wait_timeout_ms = float(wait_timeout_ms)
    o.reliable_interval = int(reliable_interval)
    o.reliable_delta = float(reliable_delta)
    o.phase_timing = 1 if phase_timing else 0
    o.test_stall = 1 if test_stall else 0
    o.preconditioner = int(preconditioner)
    o.trace_iteration = int(trace_iteration)
    o.smoother = int(smoother)
    o.fallback = 1 if fallback else 0
    o.batch_part_nodes = int(batch_part_nodes)
    return o


class Context:
    """A pg_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        st = self.L.pg_create(int(device), C.byref(h))
        if st != PG_OK:
            raise PlateGPUError(st, self.L.pg_last_error(None).decode())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.pg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != PG_OK:
            raise PlateGPUError(st, self.L.pg_last_error(self.h).decode())

    def solve(self, prob: Problem, opts: PgOptions):
        x = np.zeros(prob.F.size, np.float64)
        info = PgInfo()
        st = self.L.pg_solve(self.h, C.byref(prob.struct), C.byref(opts), _ptr(x), C.byref(info))
        self._check(st)
        return x, info

    def solve_load_cases(self, prob: Problem, F, opts: PgOptions, cases_per_launch: int = 0):
        """pg_solve_load_cases: F [k][3 Nn] loads of one plate -> (x [k][3 Nn]
        FP64, list of k PgInfo)."""
        F = np.ascontiguousarray(F, np.float32)
        if F.ndim != 2:
            raise ValueError("F must be [cases][3 * node_count]")
        k = F.shape[0]
        x = np.zeros(F.shape, np.float64)
        infos = (PgInfo * k)()
        st = self.L.pg_solve_load_cases(self.h, C.byref(prob.struct), k, _ptr(F), C.byref(opts),
                                        int(cases_per_launch), _ptr(x), infos)
        self._check(st)
        return x, list(infos)

    def plan(self, prob: Problem, opts: PgOptions) -> "DevicePlan":
        return DevicePlan(self, prob, opts)

    def batch(self, probs, opts: PgOptions) -> "Batch":
        return Batch(self, probs, opts)

    def solve_batch(self, probs, opts: PgOptions):
        """pg_solve_batch: plan, solve and release in one call."""
        arr = (PgProblem * len(probs))(*[p.struct for p in probs])
        xs = [np.zeros(p.F.size, np.float64) for p in probs]
        xp = (C.c_void_p * len(probs))(*[x.ctypes.data for x in xs])
        infos = (PgInfo * len(probs))()
        bi = PgBatchInfo()
        st = self.L.pg_solve_batch(self.h, arr, len(probs), C.byref(opts), C.cast(xp, C.c_void_p),
                                   C.cast(infos, C.c_void_p), C.byref(bi))
        self._check(st)
        return xs, list(infos), bi

    def moments(self, prob: Problem, x):
        """pg_moments: nodal (Mx, My, Mxy) of displacements x (FP64)."""
        x = np.ascontiguousarray(x, np.float64)
        n = int(prob.struct.node_count)
        out = [np.zeros(n, np.float64) for _ in range(3)]
        self._check(self.L.pg_moments(self.h, C.byref(prob.struct), _ptr(x), *[_ptr(o) for o in out]))
        return tuple(out)

    def apply_k(self, prob: Problem, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        self._check(self.L.pg_apply_k(self.h, C.byref(prob.struct), _ptr(x), _ptr(y)))
        return y

    def block_jacobi(self, prob: Problem):
        out = np.zeros(9 * prob.struct.node_count, np.float64)
        self._check(self.L.pg_block_jacobi(self.h, C.byref(prob.struct), _ptr(out)))
        return out

    def element_stiffness(self, prob: Problem):
        npe = prob.struct.nodes_per_element
        out = np.zeros(prob.struct.element_count * 9 * npe * npe, np.float64)
        self._check(self.L.pg_element_stiffness(self.h, C.byref(prob.struct), _ptr(out)))
        return out.reshape(prob.struct.element_count, 3 * npe, 3 * npe)

    def set_stream(self, stream_ptr: int):
        self._check(self.L.pg_set_stream(self.h, C.c_void_p(stream_ptr)))

    def clear_cache(self):
        self._check(self.L.pg_clear_cache(self.h))


class Batch:
    """A pg_batch: independent plates solved together by one persistent
    launch (teams of blocks, one queue of plates per team)."""

    def __init__(self, ctx: Context, probs, opts: PgOptions):
        self.ctx = ctx
        self.probs = list(probs)  # keeps the host arrays alive while planning
        arr = (PgProblem * len(self.probs))(*[p.struct for p in self.probs])
        h = C.c_void_p()
        ctx._check(ctx.L.pg_batch_create(ctx.h, arr, len(self.probs), C.byref(opts), C.byref(h)))
        self.h = h

    def solve(self, opts: PgOptions, F=None, want_x: bool = True):
        """Returns (list of x or None, list of PgInfo, PgBatchInfo); F: optional
        list of new loads (None entries keep a plate's load)."""
        n = len(self.probs)
        fp = None
        keep = []
        if F is not None:
            arrs = [None if f is None else np.ascontiguousarray(f, np.float32) for f in F]
            keep = arrs
            fp = (C.c_void_p * n)(*[None if a is None else a.ctypes.data for a in arrs])
        xs = [np.zeros(p.F.size, np.float64) for p in self.probs] if want_x else None
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in xs]) if want_x else None
        infos = (PgInfo * n)()
        bi = PgBatchInfo()
        st = self.ctx.L.pg_batch_solve(self.h, C.byref(opts), None if fp is None else C.cast(fp, C.c_void_p),
                                       None if xp is None else C.cast(xp, C.c_void_p),
                                       C.cast(infos, C.c_void_p), C.byref(bi))
        del keep
        self.ctx._check(st)
        return xs, list(infos), bi

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.pg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_schedule(node_counts, sms: int, cap: int) -> dict:
    """pg_batch_schedule (host only): per plate its phase, team size and
    team within the phase; per phase its grid."""
    nc = np.ascontiguousarray(node_counts, np.uint32)
    n = nc.size
    phase, size, team, grid = (np.zeros(n, np.int32) for _ in range(4))
    phases = C.c_int32()
    st = load().pg_batch_schedule(_ptr(nc), n, int(sms), int(cap), _ptr(phase), _ptr(size),
                                  _ptr(team), _ptr(grid), C.byref(phases))
    if st != PG_OK:
        raise PlateGPUError(st, "batch schedule failed")
    return {"plate_phase": phase, "plate_size": size, "plate_team": team,
            "phase_grid": grid[:phases.value].copy(), "phases": phases.value}


def partition_nodes(nodes, ctas: int) -> np.ndarray:
    """pg_partition_nodes (host only): the part (thread block) of each node
    in a solve over `ctas` blocks."""
    xy = np.ascontiguousarray(nodes, np.float32).reshape(-1)
    n = xy.size // 2
    part = np.zeros(n, np.int32)
    st = load().pg_partition_nodes(_ptr(xy), n, int(ctas), _ptr(part))
    if st != PG_OK:
        raise PlateGPUError(st, "partition failed")
    return part


class DevicePlan:
    """A pg_plan: the partition and device copies of one mesh, for repeated
    device-resident solves with new loads."""

    def __init__(self, ctx: Context, prob: Problem, opts: PgOptions):
        self.ctx = ctx
        self.prob = prob  # keeps the host arrays alive while the plan is built
        h = C.c_void_p()
        ctx._check(ctx.L.pg_plan_create(ctx.h, C.byref(prob.struct), C.byref(opts), C.byref(h)))
        self.h = h

    def solve_device(self, opts: PgOptions, F_dev_ptr: int, x_dev_ptr: int) -> PgInfo:
        info = PgInfo()
        st = self.ctx.L.pg_plan_solve_device(self.h, C.byref(opts), C.c_void_p(F_dev_ptr),
                                             C.c_void_p(x_dev_ptr), C.byref(info))
        self.ctx._check(st)
        return info

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.pg_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Net:
    """A pg_net: the learned preconditioner's U-Net on a height x width grid."""

    def __init__(self, ctx: Context, height: int, width: int, seed: int = 1):
        self.ctx = ctx
        h = C.c_void_p()
        ctx._check(ctx.L.pg_net_create(ctx.h, int(height), int(width), C.c_uint64(int(seed)), C.byref(h)))
        self.h = h
        self.height, self.width = int(height), int(width)

    @property
    def param_count(self) -> int:
        return int(self.ctx.L.pg_net_param_count(self.h))

    def set_params(self, params=None, scales=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        if p is not None and p.size != self.param_count:
            raise ValueError(f"expected {self.param_count} parameters, got {p.size}")
        s = None if scales is None else np.ascontiguousarray(scales, np.float32)
        if s is not None and s.size != 6:
            raise ValueError("scales: 6 values")
        self.ctx._check(self.ctx.L.pg_net_set_params(self.h, _ptr(p), _ptr(s)))

    def get_params(self):
        p = np.zeros(self.param_count, np.float32)
        s = np.zeros(6, np.float32)
        self.ctx._check(self.ctx.L.pg_net_get_params(self.h, _ptr(p), _ptr(s)))
        return p, s

    def forward(self, batch: int, in_dev: int, out_dev: int):
        self.ctx._check(self.ctx.L.pg_net_forward(self.h, int(batch), C.c_void_p(in_dev), C.c_void_p(out_dev)))

    def backward(self, batch: int, gout_dev: int, gin_dev=None, want_params: bool = True):
        g = np.zeros(self.param_count, np.float32) if want_params else None
        self.ctx._check(self.ctx.L.pg_net_backward(self.h, int(batch), C.c_void_p(gout_dev),
                                                   None if gin_dev is None else C.c_void_p(gin_dev), _ptr(g)))
        return g

    def adam_step(self, grads, lr: float):
        g = np.ascontiguousarray(grads, np.float32)
        self.ctx._check(self.ctx.L.pg_net_adam_step(self.h, _ptr(g), C.c_float(lr)))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.pg_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PG_LOSS_ENERGY, PG_LOSS_SCALED_L2, PG_LOSS_SMOOTHED_ENERGY = 0, 1, 2


def train_options(epochs=20, batch=32, lr=1e-3, cosine=True, seed=1, val_count=0,
                  set_scales=True, loss=PG_LOSS_ENERGY) -> PgTrainOptions:
    o = PgTrainOptions()
    load().pg_train_options_default(C.byref(o))
    o.epochs, o.batch, o.lr = int(epochs), int(batch), float(lr)
    o.cosine, o.seed, o.val_count = int(bool(cosine)), int(seed), int(val_count)
    o.set_scales = int(bool(set_scales))
    o.loss = int(loss)
    return o


class Learned:
    """A pg_learned: flexible PCG with the network as the coarse correction
    of a two-level preconditioner, on one plan."""

    def __init__(self, plan: "DevicePlan", net: Net, node_pixel):
        self.ctx, self.plan, self.net = plan.ctx, plan, net
        npx = np.ascontiguousarray(node_pixel, np.int32)
        h = C.c_void_p()
        self.ctx._check(self.ctx.L.pg_learned_create(plan.h, net.h, _ptr(npx), C.byref(h)))
        self.h = h
        self.n = 3 * int(plan.prob.struct.node_count)

    def make_pairs(self, count, F_dev, xstar_dev, xk_dev, R_dev, E_dev):
        self.ctx._check(self.ctx.L.pg_learned_make_pairs(
            self.h, int(count), C.c_void_p(F_dev), C.c_void_p(xstar_dev),
            None if xk_dev is None else C.c_void_p(xk_dev), C.c_void_p(R_dev), C.c_void_p(E_dev)))

    def train(self, count, R_dev, E_dev, opts: PgTrainOptions):
        info = PgTrainInfo()
        self.ctx._check(self.ctx.L.pg_learned_train(self.h, int(count), C.c_void_p(R_dev), C.c_void_p(E_dev),
                                                    C.byref(opts), C.byref(info)))
        return info

    def loss(self, count, R_dev, E_dev):
        out = np.zeros(int(count), np.float64)
        self.ctx._check(self.ctx.L.pg_learned_loss(self.h, int(count), C.c_void_p(R_dev), C.c_void_p(E_dev),
                                                   _ptr(out)))
        return out

    def solve_device(self, opts: PgOptions, F_dev: int, x_dev: int, mode: int = LEARNED_NETWORK):
        info, stats = PgInfo(), PgLearnedStats()
        self.ctx._check(self.ctx.L.pg_learned_solve_device(self.h, C.byref(opts), int(mode), C.c_void_p(F_dev),
                                                           C.c_void_p(x_dev), C.byref(info), C.byref(stats)))
        return info, stats

    def solve(self, opts: PgOptions, F, mode: int = LEARNED_NETWORK):
        F = np.ascontiguousarray(F, np.float32)
        x = np.zeros(self.n, np.float64)
        info, stats = PgInfo(), PgLearnedStats()
        self.ctx._check(self.ctx.L.pg_learned_solve(self.h, C.byref(opts), int(mode), _ptr(F), _ptr(x),
                                                    C.byref(info), C.byref(stats)))
        return x, info, stats

    def apply_k(self, x):
        """K x (FP32) by the operator the flexible PCG applies."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros(self.n, np.float32)
        self.ctx._check(self.ctx.L.pg_learned_apply_k(self.h, _ptr(x), _ptr(y)))
        return y

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.pg_learned_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
