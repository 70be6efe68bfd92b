"""The strip partition of the persistent kernel's plan (host logic, no GPU):
pg_partition_nodes against the numpy model the two-level tests use
(two_level_ref.strip_partition: nodes sorted by (y, x, id) into strips,
each strip sorted by (x, y, id) and cut into its blocks).  The partition
decides the parts, the coarse aggregates and so the iterates, so the C++
sort must order ties and signed zeros exactly as the model does.
"""
import numpy as np
import pytest

from plategpu import _lib, mesher, workloads
from two_level_ref import strip_partition


def _check(xy, G):
    xy = np.asarray(xy, np.float32).reshape(-1, 2)
    got = _lib.partition_nodes(xy, G)
    want = strip_partition(xy.astype(np.float64), min(G, xy.shape[0]))
    np.testing.assert_array_equal(got, want)
    assert got.min() == 0 and got.max() == min(G, xy.shape[0]) - 1


MESHES = {
    "plate_q4_32": lambda: workloads.plate_q4_32().mesh.nodes,
    "plate_q4_141": lambda: workloads.plate_q4_141().mesh.nodes,
    "jittered_dkt": lambda: mesher.split_triangle_mesh(10, 10, 30, 30, jitter=0.2, seed=6).nodes,
    "plate_holes_dkt": lambda: workloads.plate_holes_dkt().mesh.nodes,
}


@pytest.mark.parametrize("name", sorted(MESHES))
@pytest.mark.parametrize("G", [1, 2, 7, 37, 148])
def test_partition_matches_model(name, G):
    _check(MESHES[name](), G)


def test_partition_signed_zero_and_ties():
    # a grid centred on 0 with a column at -0.0 and a row at +0.0, plus
    # duplicated points (equal (x, y): ordered by node id)
    xy = np.asarray(workloads.plate_q4_32().mesh.nodes, np.float32).reshape(-1, 2).copy()
    cx, cy = np.median(xy[:, 0]), np.median(xy[:, 1])
    xy[:, 0] = -(xy[:, 0] - cx)
    xy[:, 1] = xy[:, 1] - cy
    assert np.any(np.signbit(xy[:, 0]) & (xy[:, 0] == 0))
    dup = np.concatenate([xy, xy[::7]])
    for G in (3, 16, 64):
        _check(xy, G)
        _check(dup, G)


def test_partition_random_cloud_and_clamp():
    rng = np.random.default_rng(3)
    xy = rng.random((997, 2)).astype(np.float32) * np.float32([7.0, 2.0])
    for G in (5, 148, 997, 2000):
        _check(xy, G)


def test_partition_rejects_bad_input():
    xy = np.zeros((4, 2), np.float32)
    with pytest.raises(_lib.PlateGPUError):
        _lib.partition_nodes(xy, 0)
    xy[2, 1] = np.nan
    with pytest.raises(_lib.PlateGPUError):
        _lib.partition_nodes(xy, 2)
