"""ctypes wrapper over liboracle.so, the CPU restatement of the reference solver.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, always as the checker and never as the thing
measured or shipped.  The restated reference functions are cited in
plate_oracle.c; every wrapper here names the reference function it mirrors.

Modes: REF reproduces the reference's Float32Array/JS-double arithmetic,
FP64 is the same formulas without binary32 rounding (the FP64 truth
operator).  ``truth_solve`` assembles that FP64 operator and solves it with
a sparse direct factorisation plus FP64 iterative refinement.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

REF = 0
FP64 = 1

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_I = C.c_int
_D = C.c_double
_IP = C.POINTER(C.c_int)
_DPp = C.POINTER(C.c_double)


def build() -> str:
    """Compiles liboracle.so with the committed Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "plate_oracle.c")
        ):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_q4_ke.argtypes = [_fp, _D, _D, _D, _I, _dp]
        L.or_dkt_ke.argtypes = [_fp, _D, _D, _D, _I, _dp]
        L.or_rect_dims.argtypes = [_D, _D, _D, _IP, _IP]
        L.or_rect_mesh.argtypes = [_D, _D, _I, _I, _fp, _up, _up]
        L.or_color_structured.argtypes = [_I, _I, _u8p, _up, _ip]
        L.or_color_greedy.argtypes = [_I, _I, _I, _up, _u8p, _up, _ip]
        L.or_color_greedy.restype = _I
        L.or_moments.argtypes = [_I, _I, _I, _fp, _up, _D, _D, _D, _dp, _I, _dp, _dp, _dp]
        L.or_verify_coloring.argtypes = [_I, _I, _I, _up, _u8p]
        L.or_verify_coloring.restype = _I
        L.or_all_ke.argtypes = [_I, _I, _fp, _up, _D, _D, _D, C.c_void_p, _I, _dp]
        L.or_diagonal.argtypes = [_I, _I, _I, _up, _dp, _I, _dp]
        L.or_block_diag.argtypes = [_I, _I, _I, _up, _dp, _I, _dp]
        L.or_invert_block_diag.argtypes = [_I, _dp, _u8p, _I]
        L.or_block_precond.argtypes = [_I, _dp, _dp, _dp, _I]
        L.or_constrained.argtypes = [_I, _ip, _ip, _I, _up, _u8p]
        L.or_load_vector.argtypes = [_I, _fp, _I, _dp, _dp, _I, _dp]
        L.or_apply_bcs_rhs.argtypes = [_I, _u8p, _dp]
        L.or_apply_k.argtypes = [_I, _I, _up, _dp, _I, _ip, _up, _u8p, _dp, _dp, _I]
        L.or_solve_pcg.argtypes = [_I, _I, _up, _dp, _I, _ip, _up, _u8p, _dp, _dp, _D, _I, _I,
                                   _dp, _IP, _DPp, _IP]
        L.or_solve_test_system.argtypes = [_dp, _IP, _DPp, _IP]
        L.or_assemble_coo.argtypes = [_I, _I, _I, _up, _dp, _u8p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
        L.or_assemble_coo.restype = C.c_long
        _lib = L
    return _lib


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# --- element.ts ---------------------------------------------------------------

def q4_ke(coords, E, nu, t, mode=REF):
    """computeElementStiffness (element.ts:258-483); 12x12."""
    Ke = np.zeros(144)
    lib().or_q4_ke(_f32(coords), E, nu, t, mode, Ke)
    return Ke.reshape(12, 12)


def dkt_ke(coords, E, nu, t, mode=REF):
    """computeDKTStiffness (element.ts:642-827); 9x9."""
    Ke = np.zeros(81)
    lib().or_dkt_ke(_f32(coords), E, nu, t, mode, Ke)
    return Ke.reshape(9, 9)


# --- mesher.ts / coloring.ts -------------------------------------------------

def rect_dims(width, height, target):
    nx, ny = C.c_int(), C.c_int()
    lib().or_rect_dims(width, height, target, C.byref(nx), C.byref(ny))
    return nx.value, ny.value


def rect_mesh(width, height, nx, ny):
    """generateRectangularMesh body (mesher.ts:364-439) for given nx, ny."""
    nodes = np.zeros(2 * (nx + 1) * (ny + 1), np.float32)
    elements = np.zeros(4 * nx * ny, np.uint32)
    boundary = np.zeros(2 * (nx + ny), np.uint32)
    lib().or_rect_mesh(width, height, nx, ny, nodes, elements, boundary)
    return nodes, elements, boundary


def color_structured(Ne, gridNx):
    """computeElementColoring (coloring.ts:38-81) -> (elementColors, flat, counts)."""
    ec = np.zeros(Ne, np.uint8)
    flat = np.zeros(Ne, np.uint32)
    counts = np.zeros(4, np.int32)
    lib().or_color_structured(Ne, gridNx, ec, flat, counts)
    return ec, flat, counts


def color_greedy(Nn, Ne, npe, elements):
    """computeElementColoringGreedy (coloring.ts:92-177)."""
    ec = np.zeros(Ne, np.uint8)
    flat = np.zeros(Ne, np.uint32)
    counts = np.zeros(256, np.int32)
    k = lib().or_color_greedy(Nn, Ne, npe, _u32(elements), ec, flat, counts)
    return ec, flat, counts[:k].copy()


def verify_coloring(Nn, Ne, npe, elements, element_colors):
    """verifyColoring (coloring.ts:188-225)."""
    return bool(lib().or_verify_coloring(Nn, Ne, npe, _u32(elements), _u8(element_colors)))


# --- solver.ts ----------------------------------------------------------------

def all_ke(nodes, elements, npe, E, nu, t, elem_t=None, mode=REF):
    """Ke of every element, as the reference's Ke cache holds them (solver.ts:49-77)."""
    elements = _u32(elements)
    Ne = elements.size // npe
    nd = 3 * npe
    out = np.zeros(Ne * nd * nd)
    et = None if elem_t is None else _f32(elem_t)
    lib().or_all_ke(Ne, npe, _f32(nodes), elements, E, nu, t,
                    None if et is None else et.ctypes.data_as(C.c_void_p), mode, out)
    return out.reshape(Ne, nd, nd)


def diagonal(Nn, elements, npe, ke, mode=REF):
    """computeDiagonal (solver.ts:145-177)."""
    elements = _u32(elements)
    d = np.zeros(3 * Nn)
    lib().or_diagonal(Nn, elements.size // npe, npe, elements, _f64(ke), mode, d)
    return d


def block_diag(Nn, elements, npe, ke, mode=REF):
    """computeBlockDiagonal (solver.ts:188-225); (Nn, 9)."""
    elements = _u32(elements)
    bd = np.zeros(9 * Nn)
    lib().or_block_diag(Nn, elements.size // npe, npe, elements, _f64(ke), mode, bd)
    return bd


def invert_block_diag(bd, cons, mode=REF):
    """invertBlockDiagonal (solver.ts:231-304); returns a new array."""
    out = _f64(bd).copy()
    lib().or_invert_block_diag(out.size // 9, out, _u8(cons), mode)
    return out


def block_precond(bd_inv, r, mode=REF):
    """applyBlockPreconditioner (solver.ts:313-339)."""
    z = np.zeros_like(_f64(r))
    lib().or_block_precond(z.size // 3, _f64(bd_inv), _f64(r), z, mode)
    return z


SUPPORT_TYPES = {"pinned": 0, "fixed": 1, "roller": 2}


def constrained(Nn, supports, boundary):
    """identifyConstrainedDOFs (solver.ts:92-134) as a uint8 mask of 3*Nn."""
    types = np.array([SUPPORT_TYPES[s[0]] for s in supports], np.int32)
    locs = np.array([-1 if s[1] == "all_edges" else int(s[1]) for s in supports], np.int32)
    cons = np.zeros(3 * Nn, np.uint8)
    b = _u32(boundary)
    lib().or_constrained(len(supports), types, locs, b.size, b, cons)
    return cons


def load_vector(nodes, loads, mode=REF):
    """buildLoadVector (solver.ts:363-392); loads = [((x, y), magnitude), ...]."""
    nodes = _f32(nodes)
    Nn = nodes.size // 2
    pos = np.array([p for (p, _m) in loads], np.float64).reshape(-1)
    mag = np.array([m for (_p, m) in loads], np.float64)
    F = np.zeros(3 * Nn)
    lib().or_load_vector(Nn, nodes, len(loads), _f64(pos), _f64(mag), mode, F)
    return F


def apply_k(Nn, elements, npe, ke, color_offsets, elements_by_color, cons, x, mode=REF):
    """applyGlobalK (solver.ts:422-483)."""
    y = np.zeros(3 * Nn)
    co = np.ascontiguousarray(color_offsets, np.int32)
    lib().or_apply_k(Nn, npe, _u32(elements), _f64(ke), co.size - 1, co, _u32(elements_by_color),
                     _u8(cons), _f64(x), y, mode)
    return y


def solve_pcg(Nn, elements, npe, ke, color_offsets, elements_by_color, cons, bd_inv, b, tol,
              maxit, mode=REF):
    """solvePCG with applyGlobalK and the block preconditioner (pcg.ts:98-215)."""
    x = np.zeros(3 * Nn)
    it, res, conv = C.c_int(), C.c_double(), C.c_int()
    co = np.ascontiguousarray(color_offsets, np.int32)
    lib().or_solve_pcg(Nn, npe, _u32(elements), _f64(ke), co.size - 1, co,
                       _u32(elements_by_color), _u8(cons), _f64(bd_inv), _f64(b), tol, maxit,
                       mode, x, C.byref(it), C.byref(res), C.byref(conv))
    return x, it.value, res.value, bool(conv.value)


def solve_test_system():
    """solveTestSystem (pcg.ts:221-247): known answer x = ones(10)."""
    x = np.zeros(10)
    it, res, conv = C.c_int(), C.c_double(), C.c_int()
    lib().or_solve_test_system(x, C.byref(it), C.byref(res), C.byref(conv))
    return x, it.value, res.value, bool(conv.value)


# --- postprocess.ts -------------------------------------------------------------

def moments(nodes, elements, npe, E, nu, t, x, mode=REF):
    """computeMoments (postprocess.ts:40-264): nodal (Mx, My, Mxy)."""
    nodes = _f32(nodes)
    elements = _u32(elements)
    Nn = nodes.size // 2
    out = [np.zeros(Nn) for _ in range(3)]
    lib().or_moments(Nn, elements.size // npe, npe, nodes, elements, E, nu, t, _f64(x), mode, *out)
    return tuple(out)


# --- FP64 truth -----------------------------------------------------------------

def assemble(Nn, elements, npe, ke_fp64, cons):
    """Sparse FP64 operator K_ff (+) I_cc in CSR form."""
    import scipy.sparse as sp

    elements = _u32(elements)
    Ne = elements.size // npe
    ke = _f64(ke_fp64)
    c = _u8(cons)
    m = lib().or_assemble_coo(Nn, Ne, npe, elements, ke, c, None, None, None)
    rows = np.zeros(m, np.int32)
    cols = np.zeros(m, np.int32)
    vals = np.zeros(m, np.float64)
    lib().or_assemble_coo(Nn, Ne, npe, elements, ke, c, rows.ctypes.data_as(C.c_void_p),
                          cols.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p))
    n = 3 * Nn
    return sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()


def truth_solve(Nn, elements, npe, ke_fp64, cons, F, refine=3):
    """FP64 truth x* of K_ff x = F_f (x = 0 on constrained DOFs).

    Sparse LU (SuperLU) followed by FP64 iterative refinement; returns
    (x, relative true residual)."""
    import scipy.sparse.linalg as spla

    A = assemble(Nn, elements, npe, ke_fp64, cons)
    b = _f64(F).copy()
    b[_u8(cons) != 0] = 0.0
    lu = spla.splu(A.tocsc())
    x = lu.solve(b)
    for _ in range(refine):
        r = b - A @ x
        x = x + lu.solve(r)
    bn = np.linalg.norm(b)
    rel = float(np.linalg.norm(b - A @ x) / bn) if bn > 0 else 0.0
    return x, rel


def truth_factor(Nn, elements, npe, ke_fp64, cons, refine=3):
    """truth_solve for many loads of one plate: factors the FP64 operator
    once and returns solve(F) -> (x, relative true residual)."""
    import scipy.sparse.linalg as spla

    A = assemble(Nn, elements, npe, ke_fp64, cons)
    lu = spla.splu(A.tocsc())
    mask = _u8(cons) != 0

    def solve(F):
        b = _f64(F).copy()
        b[mask] = 0.0
        x = lu.solve(b)
        for _ in range(refine):
            x = x + lu.solve(b - A @ x)
        bn = np.linalg.norm(b)
        return x, (float(np.linalg.norm(b - A @ x) / bn) if bn > 0 else 0.0)

    solve.A = A
    return solve
