"""Writes oracle_regression.npz: values of the CPU oracle on small inputs.

These pin the oracle to itself (a change to plate_oracle.c that moves any
of them fails tests/test_oracle.py).  They are NOT outputs recorded from
the reference, which cannot run here (TypeScript, no Node).
Run from the repository root:  python tests/golden/make_oracle_regression.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

q4 = np.array([0.0, 0.0, 0.7, 0.05, 0.75, 0.62, -0.02, 0.58], np.float32)
tri = np.array([0.0, 0.0, 0.9, 0.1, 0.2, 0.8], np.float32)
out = {"q4_coords": q4, "dkt_coords": tri}
for mode, name in ((O.REF, "ref"), (O.FP64, "fp64")):
    out[f"q4_ke_{name}"] = O.q4_ke(q4, 2.1e11, 0.3, 0.1, mode)
    out[f"dkt_ke_{name}"] = O.dkt_ke(tri, 2.1e11, 0.3, 0.1, mode)
# 4x4 clamped plate, point load at the centre node: ref-mode PCG
nodes, el, bnd = O.rect_mesh(10.0, 10.0, 4, 4)
ke = O.all_ke(nodes, el, 4, 2.1e11, 0.3, 0.1, mode=O.REF)
cons = O.constrained(25, [("fixed", "all_edges")], bnd)
ec, flat, counts = O.color_structured(16, 4)
co = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
bd = O.invert_block_diag(O.block_diag(25, el, 4, ke, O.REF), cons, O.REF)
F = O.load_vector(nodes, [((5.0, 5.0), 1000.0)], O.REF)
x, it, res, conv = O.solve_pcg(25, el, 4, ke, co, flat, cons, bd, F, 1e-6, 1000, O.REF)
out.update(pcg4_x=x, pcg4_iters=np.array(it), pcg4_res=np.array(res))
np.savez(os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_regression.npz"), **out)
print("wrote oracle_regression.npz; iterations", it, "residual", res)
