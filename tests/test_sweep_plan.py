"""CPU tests of how a sweep or a rolling analysis is split across devices (esrrf_sweep_plan: host
arithmetic in libesrrf, no device work), and of the gather of the sharded outputs.

The reference runs one device (LiveSRRF_CL.checkDevices picks one, LiveSRRF_CL.java:111-155); its
sweep loops over (radius, sensitivity) combinations (gui/ParametersSweep_.java:328-519) and its
rolling analysis over blocks (gui/LiveSRRF_optimised_.java:276-389), all independent.  The split
takes either the (magnification, radius) pairs (longest first onto the least-loaded device) or the
blocks (contiguous runs of balanced frame span), whichever has the smaller largest cost.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def plan(esrrf, T, mags, radii, blocks, devices, w=64, h=64, interpolation="fht"):
    return esrrf.Sweep.plan(w, h, T, mags, radii, [1, 2], blocks, devices, interpolation=interpolation)


def test_single_device_takes_everything(esrrf_mod):
    pd, bd, cost = plan(esrrf_mod, 100, [2, 4], [1.0, 2.0], [(0, 50), (50, 50)], [3])
    assert pd == [3, 3, 3, 3] and bd == [3, 3] and cost[0] > 0


def test_many_pairs_are_split_by_cost(esrrf_mod):
    """The sweep workload's 88 (M, radius) pairs... here 2 x 11 radii across 4 devices: every pair
    on exactly one device, every block on all of them, costs within 15 % of each other."""
    radii = [0.5 + 0.25 * k for k in range(11)]
    pd, bd, cost = plan(esrrf_mod, 200, [2, 4], radii, [(0, 37), (37, 64), (101, 99), (0, 100)],
                        [0, 1, 2, 3])
    assert all(d in (0, 1, 2, 3) for d in pd)
    assert bd == [-1, -1, -1, -1]
    assert max(cost) <= 1.15 * min(cost)
    # the pair costs grow with the radius: the largest pair sits alone or with the smallest ones
    assert len(set(pd)) == 4


def test_one_pair_splits_the_blocks_contiguously(esrrf_mod):
    """A rolling analysis (one pair) of 500 frames in 5 blocks of 100: blocks, not pairs, are
    split; each device's blocks are contiguous runs and the largest run is the least possible
    (two blocks on 3 or 4 devices, one block each on 5)."""
    blocks = [(100 * k, 100) for k in range(5)]
    for n_dev, most in ((4, 2), (3, 2), (5, 1), (2, 3)):
        pd, bd, cost = plan(esrrf_mod, 500, [4], [1.5], blocks, list(range(n_dev)))
        assert pd == [-1]
        assert bd == sorted(bd)  # contiguous runs in start order
        assert max(bd.count(d) for d in set(bd)) == most
        nonzero = [c for c in cost if c > 0]
        assert max(nonzero) == most / min(bd.count(d) for d in set(bd)) * min(nonzero)


def test_more_devices_than_work(esrrf_mod):
    """Two blocks and one pair on eight devices: two devices work, the rest get nothing."""
    pd, bd, cost = plan(esrrf_mod, 40, [2], [1.0], [(0, 20), (20, 20)], list(range(8)))
    assert sorted(bd) == [0, 1] and pd == [-1]
    assert sum(c > 0 for c in cost) == 2


def test_overlapping_blocks_stay_together(esrrf_mod):
    """Overlapping rolling blocks (gap < length) are cut only where the cut saves frames."""
    blocks = [(0, 100), (50, 100), (100, 100), (150, 100)]
    pd, bd, cost = plan(esrrf_mod, 250, [2], [1.5], blocks, [0, 1])
    assert bd == [0, 0, 1, 1]


def test_a_device_listed_twice_takes_two_shards(esrrf_mod):
    """Entries of the device list are shards: a device listed twice is planned like two devices
    (costs per entry), and the reported device of each unit is the ordinal."""
    radii = [0.5 + 0.25 * k for k in range(11)]
    blocks = [(0, 37), (37, 64), (101, 99), (0, 100)]
    pd2, bd2, cost2 = plan(esrrf_mod, 200, [2, 4], radii, blocks, [0, 1])
    pd, bd, cost = plan(esrrf_mod, 200, [2, 4], radii, blocks, [5, 5])
    assert cost == cost2 and bd == bd2
    assert pd == [5] * len(pd)
    blocks = [(100 * k, 100) for k in range(4)]
    pd, bd, cost = plan(esrrf_mod, 400, [4], [1.5], blocks, [0, 0])
    assert pd == [-1] and bd == [0, 0, 0, 0] and cost[0] == cost[1] > 0


def test_drift_in_a_bicubic_sweep_is_rejected(esrrf_mod):
    from esrrf import EsrrfError
    with pytest.raises(EsrrfError, match="drift"):
        esrrf_mod.Sweep(16, 16, 10, [2], [1.0], [1], [(0, 10)], interpolation="bicubic",
                        drift=(np.zeros(10), np.zeros(10)), devices=[0])


# ---------------------------------------------------------------------------------- gloo ranks


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _blocks_of_rank(bd, rank, nB):
    return [b for b in range(nB) if bd[b] == rank or bd[b] == -1]


def _rank_worker(rank, world, port, blocks, bd, raw, out):
    """One rank per device of the split: the oracle reconstruction of this rank's blocks (the
    stand-in for its device's sweep), gathered on rank 0 into the global block order."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        M = 2
        mine = _blocks_of_rank(bd, rank, len(blocks))
        interp = O.fht_interpolate(raw, M)
        part = np.zeros((len(blocks), 4, raw.shape[1] * M, raw.shape[2] * M), np.float32)
        for b in mine:
            st, ln = blocks[b]
            part[b] = O.fht_block(interp[st:st + ln], M, 1.5, 2)
        t = torch.from_numpy(part)
        gathered = [torch.zeros_like(t) for _ in range(world)] if rank == 0 else None
        dist.gather(t, gathered, dst=0)
        if rank == 0:
            full = np.zeros_like(part)
            for r in range(world):
                for b in _blocks_of_rank(bd, r, len(blocks)):
                    full[b] = gathered[r].numpy()[b]
            out["full"] = full
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_rolling_gathers_the_single_device_layout(esrrf_mod):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from esrrf import synth
    from oracle import oracle as O
    raw = synth.small_stack(77, 18, 12, 12).astype(np.float32)
    blocks = [(0, 6), (6, 5), (11, 7)]
    _, bd, _ = plan(esrrf_mod, 18, [2], [1.5], blocks, [0, 1], w=12, h=12)
    assert sorted(set(bd)) == [0, 1]
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_worker, args=(2, port, blocks, bd, raw, out), nprocs=2, join=True)
        full = out["full"]
    interp = O.fht_interpolate(raw, 2)
    for b, (st, ln) in enumerate(blocks):
        np.testing.assert_array_equal(full[b], O.fht_block(interp[st:st + ln], 2, 1.5, 2))


def test_non_finite_or_huge_drift_is_rejected(esrrf_mod):
    """Shifts become integer tile offsets in the kernels: NaN, infinite or beyond 1e6 pixels is an
    error before any device work (validation is host arithmetic, as esrrf_sweep_plan runs it)."""
    import ctypes

    from esrrf import EsrrfError, _lib
    for bad in (np.nan, np.inf, 2e6):
        sw = esrrf_mod.Sweep.__new__(esrrf_mod.Sweep)
        dx = np.zeros(10, np.float32)
        dx[3] = bad
        p = sw._params(16, 16, 10, [2], [1.0], [1], [(0, 10)], True, -1, "fht", (np.zeros(10), dx), None)
        with pytest.raises(EsrrfError, match="finite"):
            _lib.check(None, esrrf_mod.lib().esrrf_sweep_plan(ctypes.byref(p), None, None, None), sweep=True)
