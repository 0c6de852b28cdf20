"""GPU tests of the batched sweep / rolling analysis (esrrf_sweep_*): every (magnification,
radius, sensitivity, block) output must match the oracle's single-block FHT reconstruction of
that block within 1e-4 of each slice's dynamic range, and graph replays must be reproducible."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4


def test_sweep_matches_per_block_oracle(esrrf_mod, oracle_mod):
    from esrrf import synth
    raw = synth.small_stack(51, 30, 32, 32, emitters=16)
    mags, radii, sens = [2, 3], [1.0, 1.5, 2.5], [1, 2, 3]
    blocks = [(0, 10), (10, 20), (0, 20), (5, 7)]   # uneven and overlapping
    sw = esrrf_mod.Sweep(32, 32, 30, mags, radii, sens, blocks)
    try:
        res = sw.run(raw)
        assert len(res) == len(mags) * len(radii) * len(sens) * len(blocks)
        assert sw.launch_count() > 0
        interp = {M: oracle_mod.fht_interpolate(raw.astype(np.float32), M) for M in mags}
        for (M, r, S, (st, ln)), got in res.items():
            ref = oracle_mod.fht_block(interp[M][st:st + ln], M, r, S)
            for k in range(4):
                assert rel_err(got[k], ref[k]) < TOL, (M, r, S, st, ln, k)
        again = sw.run(raw)  # second run replays the captured graph
        for key in res:
            np.testing.assert_array_equal(again[key], res[key])
    finally:
        sw.release()


def test_rolling_matches_engine_blocks(esrrf_mod):
    """Rolling analysis over uneven blocks equals running the engine block by block."""
    from esrrf import synth
    raw = synth.small_stack(52, 40, 24, 24)
    blocks = [(0, 13), (13, 27), (3, 30)]
    res = esrrf_mod.rolling(raw, 4, 1.5, 2, blocks)
    for (st, ln) in blocks:
        eng = esrrf_mod.LiveSRRF_CL()
        eng.initialise(24, 24, 4, 1.5, 2, ln, ln)
        try:
            eng.resetFramePosition()
            eng.calculateSRRF(raw[st:st + ln])
            ref = eng.readSRRFbuffer()
        finally:
            eng.release()
        for k in range(4):
            assert rel_err(res[(st, ln)][k], ref[k]) < TOL, (st, ln, k)


def test_bicubic_sweep_matches_per_block_oracle(esrrf_mod, oracle_mod):
    """The bicubic sweep (ParametersSweep_ with "Use FHT interpolation" off: the bicubic path with
    MP correction) against the oracle's single-block bicubic reconstruction of every block, on a
    frame whose size is no multiple of the kernel's 32 x 8 cell tiles; graph replays reproduce."""
    from esrrf import synth
    raw = synth.small_stack(53, 24, 29, 37, emitters=16)
    mags, radii, sens = [2, 3, 4], [1.0, 2.0], [1, 2]
    blocks = [(0, 9), (9, 15), (3, 12)]
    sw = esrrf_mod.Sweep(37, 29, 24, mags, radii, sens, blocks, interpolation="bicubic")
    try:
        res = sw.run(raw)
        assert len(res) == len(mags) * len(radii) * len(sens) * len(blocks)
        for (M, r, S, (st, ln)), got in res.items():
            ref = oracle_mod.bic_block(raw[st:st + ln].astype(np.float32), M, r, S, mp_correction=True)
            for k in range(4):
                assert rel_err(got[k], ref[k]) < TOL, (M, r, S, st, ln, k)
        again = sw.run(raw)
        for key in res:
            np.testing.assert_array_equal(again[key], res[key])
    finally:
        sw.release()


def test_bicubic_rolling_matches_engine_blocks(esrrf_mod):
    """Rolling analysis on the bicubic path equals running the engine (bicubic, MP correction)
    block by block."""
    from esrrf import synth
    raw = synth.small_stack(54, 30, 24, 40)
    blocks = [(0, 11), (11, 19), (5, 20)]
    res = esrrf_mod.rolling(raw, 4, 1.5, 2, blocks, interpolation="bicubic")
    for (st, ln) in blocks:
        eng = esrrf_mod.LiveSRRF_CL()
        eng.initialise(40, 24, 4, 1.5, 2, ln, ln, doMPmapCorrection=True, doFHTinterpolation=False)
        try:
            eng.resetFramePosition()
            assert not eng.calculateSRRF(raw[st:st + ln])
            ref = eng.readSRRFbuffer().copy()
        finally:
            eng.release()
        for k in range(4):
            assert rel_err(res[(st, ln)][k], ref[k]) < TOL, (st, ln, k)


def _shards_vs_single(esrrf_mod, raw, mags, radii, sens, blocks, by, **kw):
    """The same sweep on one device and split into shards of a device listed twice (each shard
    with its own frame range, stream and graph, gathered into the caller's layout); ``by``: the
    split the planner must choose ("pairs" or "blocks")."""
    h, w = raw.shape[1:]
    pd, bd, _ = esrrf_mod.Sweep.plan(w, h, raw.shape[0], mags, radii, sens, blocks, [0, 0],
                                     interpolation=kw.get("interpolation", "fht"))
    if by == "pairs":
        assert bd == [-1] * len(blocks) and pd == [0] * len(pd)
    else:
        assert pd == [-1] * len(pd) and bd == [0] * len(blocks)
    one = esrrf_mod.Sweep(w, h, raw.shape[0], mags, radii, sens, blocks, **kw)
    two = esrrf_mod.Sweep(w, h, raw.shape[0], mags, radii, sens, blocks, devices=[0, 0], **kw)
    try:
        assert one.shard_count() == 1 and two.shard_count() == 2
        ref = one.run(raw)
        got = two.run(raw)
        again = two.run(raw)
    finally:
        one.release()
        two.release()
    assert got.keys() == ref.keys()
    for key in ref:
        np.testing.assert_array_equal(again[key], got[key])
        for k in range(4):
            assert rel_err(got[key][k], ref[key][k]) < 1e-6, (key, k, rel_err(got[key][k], ref[key][k]))


def test_sweep_split_by_pairs_gathers_the_single_device_layout(esrrf_mod):
    """The multi-device split by (magnification, radius) pairs, run as two shards on this device:
    every output lands in its place of the global layout, equal to the unsplit sweep."""
    from esrrf import synth
    raw = synth.small_stack(55, 24, 32, 40, emitters=16)
    _shards_vs_single(esrrf_mod, raw, [2, 3], [1.0, 1.5, 2.5], [1, 2], [(0, 10), (10, 14), (5, 7)], "pairs")


def test_rolling_split_by_blocks_gathers_the_single_device_layout(esrrf_mod):
    """The split by contiguous runs of blocks (one pair): each shard copies only its frame range
    and its part of the per-frame drift; FHT with drift and bicubic without."""
    from esrrf import synth
    raw = synth.small_stack(56, 40, 32, 32, emitters=16)
    blocks = [(0, 10), (10, 10), (20, 10), (30, 10)]
    rng = np.random.default_rng(7)
    drift = (rng.uniform(-1.2, 1.2, 40).astype(np.float32), rng.uniform(-1.2, 1.2, 40).astype(np.float32))
    _shards_vs_single(esrrf_mod, raw, [4], [1.5], [2], blocks, "blocks", drift=drift)
    _shards_vs_single(esrrf_mod, raw, [3], [1.5], [1], blocks, "blocks", interpolation="bicubic")


def test_pinned_output_is_filled_during_the_run(esrrf_mod):
    """A one-device sweep given a pinned host buffer copies each (magnification, radius) pair's
    outputs out while the next pairs compute (copies inside the captured graph): the same results
    as a pageable buffer, on the first run, on graph replays and with a second pinned buffer."""
    import torch

    from esrrf import synth
    raw = synth.small_stack(57, 20, 24, 32, emitters=12)
    for interp in ("fht", "bicubic"):
        sw = esrrf_mod.Sweep(32, 24, 20, [2, 3], [1.0, 2.0], [1, 2], [(0, 12), (4, 16)], interpolation=interp)
        try:
            ref = {k: v.copy() for k, v in sw.run(raw).items()}
            bufs = [torch.full((sw.total,), float("nan"), dtype=torch.float32).pin_memory() for _ in range(2)]
            for buf in (bufs[0], bufs[0], bufs[1]):
                buf.fill_(float("nan"))
                got = sw.run(raw, out=buf.numpy())
                assert got.keys() == ref.keys()
                for key in ref:
                    np.testing.assert_array_equal(got[key], ref[key], err_msg=f"{interp} {key}")
        finally:
            sw.release()


def test_stack_of_the_wrong_shape_is_rejected(esrrf_mod):
    from esrrf import EsrrfError, synth
    raw = synth.small_stack(58, 10, 16, 20, emitters=4)
    sw = esrrf_mod.Sweep(20, 16, 10, [2], [1.5], [1], [(0, 10)])
    try:
        with pytest.raises(EsrrfError, match="stack must be"):
            sw.run(raw[:9])
        with pytest.raises(EsrrfError, match="stack must be"):
            sw.run(raw.transpose(0, 2, 1))
        assert len(sw.run(raw)) == 1
    finally:
        sw.release()
