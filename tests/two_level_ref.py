"""CPU model of the two-level preconditioner (test helper).

Restates, in numpy, the coarse space the library builds: the strip
partition of the nodes into G parts (one aggregate each), the three
rigid-body modes per aggregate (w = 1; w = dy, thx = 1/h; w = dx,
thy = -1/h about the aggregate centre, h its size), P with constrained rows
removed, A_c = P^T A P, and additive two-level PCG with
M^-1 = M_bj^-1 + P A_c^-1 P^T, driven by textbook PCG.
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


def two_level_pcg(A, b, bd_inv, P, tol, maxit=20000):
    """Textbook PCG, stop on ||r|| / ||b|| < tol; returns (x, iterations)."""
    Nn = bd_inv.size // 9
    Bi = bd_inv.reshape(Nn, 3, 3)
    Ac = (P.T @ A @ P).toarray()
    Aci = np.linalg.inv(Ac)

    def M(r):
        z = np.einsum("nij,nj->ni", Bi, r.reshape(Nn, 3)).reshape(-1)
        return z + P @ (Aci @ (P.T @ r))

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
