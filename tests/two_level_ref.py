"""CPU model of the two-level preconditioner and the Chebyshev smoother
(test helper).

Restates, in numpy, the coarse space the library builds: the strip
partition of the nodes into G parts (one aggregate each), the three
rigid-body modes per aggregate (w = 1; w = dy, thx = 1/h; w = dx,
thy = -1/h about the aggregate centre, h its size), P with constrained rows
removed, A_c = P^T A P, and additive two-level PCG with
M^-1 = S + P A_c^-1 P^T, driven by textbook PCG.  S is block Jacobi
(S = D^-1) or the degree-2 Chebyshev smoother S = a D^-1 - b D^-1 A D^-1
whose coefficients come from a power-iteration estimate of
lambda_max(D^-1 A) (the library's start vector and iteration count).
"""
import numpy as np
import scipy.sparse as sp


def strip_partition(xy, G):
    Nn = xy.shape[0]
    W, H = np.ptp(xy[:, 0]), np.ptp(xy[:, 1])
    R = max(1, min(G, int(round(np.sqrt(G * H / max(W, 1e-30))))))
    ids = np.lexsort((np.arange(Nn), xy[:, 0], xy[:, 1]))
    part = np.zeros(Nn, np.int64)
    p = start = done = 0
    for s in range(R):
        blocks = G // R + (1 if s < G % R else 0)
        done += blocks
        end = Nn * done // G
        seg = ids[start:end]
        seg = seg[np.lexsort((seg, xy[seg, 1], xy[seg, 0]))]
        L = len(seg)
        for b in range(blocks):
            part[seg[L * b // blocks: L * (b + 1) // blocks]] = p
            p += 1
        start = end
    return part


def coarse_basis(xy, cons, part, G):
    n = 3 * xy.shape[0]
    rows, cols, vals = [], [], []
    for g in range(G):
        nodes = np.where(part == g)[0]
        c = xy[nodes].mean(axis=0)
        h = max(np.ptp(xy[nodes, 0]), np.ptp(xy[nodes, 1]))
        ih = 1.0 / h if h > 0 else 1.0
        for nd in nodes:
            dx, dy = (xy[nd] - c) * ih
            for m, ent in enumerate(([(0, 1.0)], [(0, dy), (1, ih)], [(0, dx), (2, -ih)])):
                for d, v in ent:
                    if not cons[3 * nd + d]:
                        rows.append(3 * nd + d)
                        cols.append(3 * g + m)
                        vals.append(v)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, 3 * G))


def lambda_max_power(A, bd_inv, cons, iters=30):
    """|D^-1 A x| after `iters` normalised power steps from the library's
    start vector x_i = 1 + 0.5 sin(0.7 i) (0 on constrained DOFs)."""
    Nn = bd_inv.size // 9
    Bi = bd_inv.reshape(Nn, 3, 3)
    i = np.arange(3 * Nn)
    x = np.where(np.asarray(cons) != 0, 0.0, 1.0 + 0.5 * np.sin(0.7 * i))
    lam = 1.0
    for _ in range(iters):
        y = np.einsum("nij,nj->ni", Bi, (A @ x).reshape(Nn, 3)).reshape(-1)
        lam = np.linalg.norm(y)
        x = y / lam
    return lam


def chebyshev2(lam):
    """(a, b) of S = a D^-1 - b D^-1 A D^-1: two Chebyshev steps for D^-1 A
    on [hi / 20, hi], hi = 1.1 lam."""
    hi = 1.1 * lam
    lo = hi / 20.0
    theta, delta = 0.5 * (hi + lo), 0.5 * (hi - lo)
    sigma = theta / delta
    rho0 = 1.0 / sigma
    rho1 = 1.0 / (2.0 * sigma - rho0)
    return (1.0 + rho1 * rho0) / theta + 2.0 * rho1 / delta, 2.0 * rho1 / (delta * theta)


def two_level_pcg(A, b, bd_inv, P, tol, maxit=20000, cheb=None):
    """Textbook PCG with M^-1 = S (+ P A_c^-1 P^T when P is given), stop on
    ||r|| / ||b|| < tol; cheb = (a, b) selects the Chebyshev smoother.
    Returns (x, iterations)."""
    Nn = bd_inv.size // 9
    Bi = bd_inv.reshape(Nn, 3, 3)
    Aci = None if P is None else np.linalg.inv((P.T @ A @ P).toarray())

    def D(v):
        return np.einsum("nij,nj->ni", Bi, v.reshape(Nn, 3)).reshape(-1)

    def M(r):
        t = D(r)
        z = t if cheb is None else cheb[0] * t - cheb[1] * D(A @ t)
        return z if P is None else z + P @ (Aci @ (P.T @ r))

    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = z.copy()
    rz = r @ z
    bn = np.linalg.norm(b)
    for it in range(maxit):
        Ap = A @ p
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        if np.linalg.norm(r) / bn < tol:
            return x, it + 1
        z = M(r)
        rzn = r @ z
        p = z + rzn / rz * p
        rz = rzn
    return x, maxit
