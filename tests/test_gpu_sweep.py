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
