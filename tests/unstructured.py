"""Unstructured triangle meshes for the tests: plates with holes from
plategpu.workloads (Delaunay triangles, shuffled node numbers), standing in
for the reference's constrained-Delaunay meshes (mesher-unstructured.ts:36-76)."""
from plategpu.workloads import plate_holes_dkt, plate_with_holes


def workload(h=0.25, seed=3, q=4e3, t=0.1, rotate=True):
    """Clamped outer edges, free hole edges, uniform pressure q plus two
    point loads; per-element thickness varying smoothly across the plate."""
    return plate_holes_dkt(h=h, seed=seed, q=q, t=t, rotate=rotate)


__all__ = ["plate_with_holes", "workload"]
