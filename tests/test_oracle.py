"""The CPU oracle against the reference's known answers and plate theory.

The reference ships no recorded outputs, so the oracle is pinned by its
known-answer system (pcg.ts:221-247), its element checks (element.ts:568-597),
verifyColoring (coloring.ts:188-225), classical plate coefficients, FP64
self-consistency, and regression fixtures of its own values.
"""
import json
import os

import numpy as np
import pytest

from conftest import rel_err

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def known():
    with open(os.path.join(GOLD, "known_answers.json")) as f:
        return json.load(f)


def test_pcg_known_answer(oracle):
    kat = known()["pcg_tridiag"]
    x, it, res, conv = oracle.solve_test_system()
    assert conv is kat["expected_converged"]
    np.testing.assert_allclose(x, kat["expected_x"], rtol=0, atol=1e-6)
    assert it <= kat["max_iterations"]


@pytest.mark.parametrize("mode", [0, 1])
def test_q4_element_checks(oracle, mode):
    rng = np.random.default_rng(4)
    for _ in range(20):
        base = np.array([0, 0, 1, 0, 1, 1, 0, 1], np.float64)
        c = (base + rng.uniform(-0.15, 0.15, 8)).astype(np.float32)
        K = oracle.q4_ke(c, 2.1e11, 0.3, rng.uniform(0.02, 0.3), mode)
        assert np.all(np.diag(K) > 0)  # isPositiveSemiDefinite (element.ts:589-597)
        assert np.max(np.abs(K - K.T)) <= 1e-6 * np.max(np.abs(K))  # isSymmetric
        ev = np.linalg.eigvalsh(K.astype(np.float64))
        assert ev.min() > -1e-7 * ev.max()
        # rigid translation in w carries no energy
        u = np.zeros(12)
        u[0::3] = 1.0
        assert np.linalg.norm(K @ u) <= 1e-9 * np.linalg.norm(K)


def test_dkt_element_checks(oracle):
    rng = np.random.default_rng(5)
    for _ in range(20):
        c = (np.array([0, 0, 1, 0, 0, 1]) + rng.uniform(-0.2, 0.2, 6)).astype(np.float32)
        K = oracle.dkt_ke(c, 2.1e11, 0.3, 0.1, 1)
        assert np.max(np.abs(K - K.T)) <= 1e-12 * np.max(np.abs(K))
        assert np.all(np.diag(K) >= 0)
        assert np.linalg.eigvalsh(K).min() > -1e-9 * np.abs(K).max()


def test_dkt_degenerate_is_zero(oracle):
    c = np.array([0, 0, 1, 1, 2, 2], np.float32)  # collinear: area 0
    assert np.all(oracle.dkt_ke(c, 2.1e11, 0.3, 0.1, 0) == 0)


def test_ref_mode_rounds_to_float32(oracle):
    c = np.array([0, 0, 0.3, 0, 0.3, 0.2, 0, 0.2], np.float32)
    K = oracle.q4_ke(c, 2.1e11, 0.3, 0.1, 0)
    assert np.all(K.astype(np.float32).astype(np.float64) == K)
    K64 = oracle.q4_ke(c, 2.1e11, 0.3, 0.1, 1)
    assert rel_err(K, K64) < 1e-6


def test_regression_fixtures(oracle):
    g = np.load(os.path.join(GOLD, "oracle_regression.npz"))
    for name in ("ref", "fp64"):
        mode = 0 if name == "ref" else 1
        np.testing.assert_array_equal(oracle.q4_ke(g["q4_coords"], 2.1e11, 0.3, 0.1, mode),
                                      g[f"q4_ke_{name}"])
        np.testing.assert_array_equal(oracle.dkt_ke(g["dkt_coords"], 2.1e11, 0.3, 0.1, mode),
                                      g[f"dkt_ke_{name}"])
    nodes, el, bnd = oracle.rect_mesh(10.0, 10.0, 4, 4)
    ke = oracle.all_ke(nodes, el, 4, 2.1e11, 0.3, 0.1, mode=0)
    cons = oracle.constrained(25, [("fixed", "all_edges")], bnd)
    ec, flat, counts = oracle.color_structured(16, 4)
    co = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    bd = oracle.invert_block_diag(oracle.block_diag(25, el, 4, ke, 0), cons, 0)
    F = oracle.load_vector(nodes, [((5.0, 5.0), 1000.0)], 0)
    x, it, res, conv = oracle.solve_pcg(25, el, 4, ke, co, flat, cons, bd, F, 1e-6, 1000, 0)
    np.testing.assert_array_equal(x, g["pcg4_x"])
    assert it == int(g["pcg4_iters"])


def _udl_plate(oracle, nx, support):
    nodes, el, bnd = oracle.rect_mesh(10.0, 10.0, nx, nx)
    Nn = (nx + 1) ** 2
    ke = oracle.all_ke(nodes, el, 4, 2.1e11, 0.3, 0.01, mode=1)
    cons = oracle.constrained(Nn, [(support, "all_edges")], bnd)
    h = 10.0 / nx
    F = np.zeros(3 * Nn)
    for k in range(4):
        np.add.at(F, 3 * el[k::4].astype(np.int64), 1000.0 * h * h / 4)
    F[cons != 0] = 0
    x, rel = oracle.truth_solve(Nn, el, 4, ke, cons, F)
    D = 2.1e11 * 0.01 ** 3 / (12 * (1 - 0.09))
    return x[0::3].max() / (1000.0 * 10.0 ** 4 / D), rel


def test_kirchhoff_coefficients(oracle):
    """Thin plate (t = 10 mm, a/t = 1000): Q4 Mindlin approaches Kirchhoff."""
    k = known()["kirchhoff_square_plate_udl"]
    c_ss, rel = _udl_plate(oracle, 48, "pinned")
    assert rel < 1e-7  # a/t = 1000 makes K very ill-conditioned
    assert abs(c_ss - k["simply_supported_c"]) / k["simply_supported_c"] < 0.02
    c_cl, _ = _udl_plate(oracle, 48, "fixed")
    assert abs(c_cl - k["clamped_c"]) / k["clamped_c"] < 0.03


def test_fp64_pcg_agrees_with_direct(oracle):
    nodes, el, bnd = oracle.rect_mesh(10.0, 10.0, 12, 12)
    Nn = 169
    ke = oracle.all_ke(nodes, el, 4, 2.1e11, 0.3, 0.1, mode=1)
    cons = oracle.constrained(Nn, [("pinned", "all_edges")], bnd)
    ec, flat, counts = oracle.color_structured(144, 12)
    co = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    bd = oracle.invert_block_diag(oracle.block_diag(Nn, el, 4, ke, 1), cons, 1)
    F = oracle.load_vector(nodes, [((5.0, 5.0), 1e4), ((2.5, 7.5), 3e3)], 1)
    F[cons != 0] = 0
    xs, _ = oracle.truth_solve(Nn, el, 4, ke, cons, F)
    x, it, res, conv = oracle.solve_pcg(Nn, el, 4, ke, co, flat, cons, bd, F, 1e-12, 5000, 1)
    assert conv
    assert rel_err(x, xs) < 1e-9
    # applyGlobalK on the solution reproduces F (FP64)
    y = oracle.apply_k(Nn, el, 4, ke, co, flat, cons, xs, 1)
    assert rel_err(y, F) < 1e-9


def test_colorings_valid(oracle):
    nodes, el, bnd = oracle.rect_mesh(10.0, 10.0, 9, 7)
    ec, flat, counts = oracle.color_structured(63, 9)
    assert oracle.verify_coloring(80, 63, 4, el, ec)
    ec2, flat2, counts2 = oracle.color_greedy(80, 63, 4, el)
    assert oracle.verify_coloring(80, 63, 4, el, ec2)
    bad = ec.copy()
    bad[1] = bad[0]
    assert not oracle.verify_coloring(80, 63, 4, el, bad)
