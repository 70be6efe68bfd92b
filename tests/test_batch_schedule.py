"""Schedule of the batched solver (host only): every plate gets a team whose
size is a power of two (or the whole device for the largest plates) large
enough for the plate's nodes to fit at `cap` nodes per block; team sizes
that cannot share the device go to separate phases (launches) whose grids
fit the device."""
import numpy as np
import pytest

from plategpu import _lib


def uneven_node_counts(count=256, seed=5):
    rng = np.random.default_rng(seed)
    sides = np.round(np.exp(rng.uniform(np.log(16), np.log(256), size=count))).astype(int)
    return (sides + 1) ** 2


@pytest.mark.parametrize("cap", [560, 470])
def test_schedule_invariants(cap):
    nodes = uneven_node_counts()
    s = _lib.batch_schedule(nodes, 148, cap)
    size, phase = s["plate_size"], s["plate_phase"]
    assert s["phases"] >= 1 and np.all(s["phase_grid"] <= 148) and np.all(s["phase_grid"] > 0)
    assert np.all((size & (size - 1) == 0) | (size == 148))
    assert np.all(size.astype(np.int64) * cap >= nodes)   # each plate's parts fit
    assert np.all((phase >= 0) & (phase < s["phases"]))
    for ph in range(s["phases"]):
        sizes = set(size[phase == ph].tolist())
        assert sum(sizes) <= 148  # one team of every size of a phase fits beside the others
        assert s["phase_grid"][ph] >= max(sizes)
    assert np.all(s["plate_team"] >= 0)


def test_schedule_single_and_small_plates():
    s = _lib.batch_schedule([289], 148, 520)
    assert s["phases"] == 1 and s["plate_size"][0] == 1 and s["phase_grid"][0] == 1
    s = _lib.batch_schedule([289] * 300, 148, 520)
    assert s["phases"] == 1 and s["phase_grid"][0] == 148  # one-block teams, all SMs busy
    assert len(set(s["plate_team"].tolist())) == 148


def test_schedule_full_device_plates_get_their_own_phase():
    s = _lib.batch_schedule([66049, 289, 4225], 148, 470)  # 257^2 needs > 128 blocks
    assert s["plate_size"][0] == 148 and s["phases"] == 2
    assert s["plate_phase"][0] != s["plate_phase"][1]


def test_schedule_rejects_a_plate_larger_than_the_device():
    with pytest.raises(_lib.PlateGPUError):
        _lib.batch_schedule([148 * 520 + 1], 148, 520)
    with pytest.raises(_lib.PlateGPUError):  # the 257^2-node plates need 447 nodes per block
        _lib.batch_schedule(uneven_node_counts(), 148, 300)


def test_shard_lpt_balances_and_covers():
    from plategpu.workloads import shard_lpt
    costs = [float(n) ** 1.5 for n in uneven_node_counts()]
    for parts in (1, 2, 4, 8):
        sh = shard_lpt(costs, parts)
        assert sorted(i for s in sh for i in s) == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in sh]
        assert max(loads) <= sum(loads) / parts + max(costs) + 1e-9  # LPT bound
    assert shard_lpt([3.0, 1.0, 2.0], 2) == [[0], [1, 2]]
