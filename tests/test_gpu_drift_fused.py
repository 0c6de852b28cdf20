"""GPU parity of vibration (drift) correction on the fused FHT-path kernel, the sweep and the
rolling analysis.

The reference applies one shift per frame (loadDriftXYGPUbuffer, LiveSRRF_CL.java:583-595, x M)
inside calculateRadialGradientConvergence (liveSRRF_noInterpolation.cl:264-268: the output pixel's
centre moves by the shift; :356-357: the intensity is getInterpolatedValue at the shifted
position).  The plugins take the shifts per block (gui/LiveSRRF_optimised_.java:283-305) or once
for the whole sweep (gui/ParametersSweep_.java:282-290, 452-454).

Checker: the reference's kernels compiled for the host (oracle/_ref) where built, else the C
restatement that is bit-identical to them on every golden fixture.  Tolerance: each slice within
1e-4 of its dynamic range.  Shifts cover negative values, values beyond one pixel, exact integers,
zero-shift frames inside a drifting block, and fractions within rounding of 0 and 1.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4


def ref_block(O, interp, M, fwhm, S, dx, dy):
    if O.ref_available():
        return O.ref_fht_block(interp, M, fwhm, S, drift_x=dx, drift_y=dy)
    return O.fht_block(interp, M, fwhm, S, drift_x=dx, drift_y=dy)


def engine_block(esrrf, frames, M, fwhm, S, dx, dy, frames_per_launch=0, kernel="fused"):
    eng = esrrf.LiveSRRF_CL()
    n = frames.shape[0]
    eng.initialise(frames.shape[-1], frames.shape[-2], M, fwhm, S, n, n, kernel=kernel,
                   framesPerLaunch=frames_per_launch)
    try:
        eng.resetFramePosition()
        eng.loadDriftXYGPUbuffer(dx, dy)
        assert not eng.calculateSRRF(frames)
        launches = eng.lastTiming()[2]
        return eng.readSRRFbuffer().copy(), launches
    finally:
        eng.release()


def shifts(rng, n):
    dx = rng.uniform(-1.6, 1.6, n).astype(np.float32)
    dy = rng.uniform(-1.6, 1.6, n).astype(np.float32)
    dx[0] = dy[0] = 0.0                       # a frame without drift inside the block
    if n > 2:
        dx[1], dy[1] = 1.0, -2.0              # exact integers
    if n > 3:
        dx[2], dy[2] = 0.24999999, -0.7500001  # x M within rounding of an integer
    return dx, dy


def check(got, ref, what):
    for k in range(4):
        e = rel_err(got[k], ref[k])
        assert e < TOL, f"{what} slice {k}: {e:.3g} of range"


def test_golden_drift_case_runs_the_fused_kernel(esrrf_mod):
    """The reference-generated fht_m4_drift fixture through the fused kernel and through the
    per-pixel kernel: both match it, and they are different code paths (their float rounding
    differs), so the fused kernel ran."""
    g = load_golden("fht_m4_drift")
    raw = g["raw"]
    M, fwhm, S = int(g["magnification"]), float(g["fwhm"]), int(g["sensitivity"])
    fused, n_fused = engine_block(esrrf_mod, raw, M, fwhm, S, g["drift_x"], g["drift_y"])
    plain, n_plain = engine_block(esrrf_mod, raw, M, fwhm, S, g["drift_x"], g["drift_y"], kernel="plain")
    assert n_fused == n_plain, (n_fused, n_plain)
    assert not np.array_equal(fused, plain)
    check(fused, g["out"], "fused")
    check(plain, g["out"], "plain")


@pytest.mark.parametrize("M,fwhm", [(2, 1.0), (4, 1.5), (3, 2.5), (5, 2.0), (4, 3.0)])
def test_fused_drift_against_reference_kernels(esrrf_mod, oracle_mod, M, fwhm):
    """Ragged frames (tiles overhang the edges), launches of 3 frames, tap boxes from 6 to 26 wide
    (and 22+ in the second compilation unit)."""
    from esrrf import synth
    rng = np.random.default_rng(100 + M)
    raw = synth.small_stack(200 + M, 8, 23, 37, emitters=14)
    dx, dy = shifts(rng, 8)
    got, _ = engine_block(esrrf_mod, raw, M, fwhm, 2, dx, dy, frames_per_launch=3)
    interp = oracle_mod.fht_interpolate(raw.astype(np.float32), M)
    check(got, ref_block(oracle_mod, interp, M, fwhm, 2, dx, dy), f"M{M} r{fwhm}")


def test_fused_drift_full_frame_size(esrrf_mod, oracle_mod):
    """512 x 512 frames at M4, radius 1.5, sensitivity 2 (the headline workload's parameters) with
    drift, launches of 2 frames."""
    from esrrf import synth
    rng = np.random.default_rng(7)
    raw = synth.make_stack("fht512", frames=4)
    dx, dy = shifts(rng, 4)
    got, _ = engine_block(esrrf_mod, raw, 4, 1.5, 2, dx, dy, frames_per_launch=2)
    interp = oracle_mod.fht_interpolate_fft(raw.astype(np.float32), 4)
    check(got, ref_block(oracle_mod, interp, 4, 1.5, 2, dx, dy), "512x512")


def test_small_frames_grouped_launch_with_drift(esrrf_mod, oracle_mod):
    """A 24 x 24 frame at M4 leaves SMs idle, so each launch splits its frames into groups across
    CTAs; with drift every group still sees its own frames' tables."""
    from esrrf import synth
    rng = np.random.default_rng(3)
    raw = synth.small_stack(31, 20, 24, 24)
    dx, dy = shifts(rng, 20)
    got, _ = engine_block(esrrf_mod, raw, 4, 1.5, 2, dx, dy, frames_per_launch=10)
    interp = oracle_mod.fht_interpolate(raw.astype(np.float32), 4)
    check(got, ref_block(oracle_mod, interp, 4, 1.5, 2, dx, dy), "grouped")


def test_sweep_with_drift_matches_per_block_oracle(esrrf_mod, oracle_mod):
    """The sweep's one shift array for the whole stack, every (M, radius, S, block)."""
    from esrrf import synth
    rng = np.random.default_rng(11)
    T = 16
    raw = synth.small_stack(57, T, 32, 32, emitters=16)
    dx, dy = shifts(rng, T)
    mags, radii, sens = [2, 4], [1.0, 2.0], [1, 3]
    blocks = [(0, 7), (7, 9), (3, 10)]
    sw = esrrf_mod.Sweep(32, 32, T, mags, radii, sens, blocks, drift=(dx, dy))
    try:
        res = sw.run(raw)
        again = sw.run(raw)
    finally:
        sw.release()
    interp = {M: oracle_mod.fht_interpolate(raw.astype(np.float32), M) for M in mags}
    for (M, r, S, (st, ln)), got in res.items():
        ref = ref_block(oracle_mod, interp[M][st:st + ln], M, r, S, dx[st:st + ln], dy[st:st + ln])
        check(got, ref, f"M{M} r{r} S{S} [{st},{st + ln})")
        np.testing.assert_array_equal(again[(M, r, S, (st, ln))], got)


def test_rolling_with_per_block_drift(esrrf_mod, oracle_mod):
    """Per-block shift arrays: non-overlapping blocks run as one sweep, overlapping ones block by
    block through the engine; both equal the oracle's block."""
    from esrrf import synth
    rng = np.random.default_rng(5)
    raw = synth.small_stack(58, 24, 28, 28)
    interp = oracle_mod.fht_interpolate(raw.astype(np.float32), 4)
    for blocks in ([(0, 10), (10, 14)], [(0, 12), (6, 12)]):
        drift = [shifts(rng, ln) for _, ln in blocks]
        res = esrrf_mod.rolling(raw, 4, 1.5, 2, blocks, drift=drift)
        for (st, ln), (dx, dy) in zip(blocks, drift):
            check(res[(st, ln)], ref_block(oracle_mod, interp[st:st + ln], 4, 1.5, 2, dx, dy), f"{blocks}")


def test_non_finite_shift_is_rejected(esrrf_mod):
    """loadDriftXYGPUbuffer with a NaN or an infinite shift is an error, and the handle keeps
    working with valid shifts afterwards."""
    from esrrf import EsrrfError, synth
    raw = synth.small_stack(81, 6, 16, 16, emitters=4)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(16, 16, 2, 1.5, 1, 6, 6)
    try:
        for bad in (np.nan, np.inf):
            dx = np.zeros(6, np.float32)
            dx[2] = bad
            with pytest.raises(EsrrfError, match="finite"):
                eng.loadDriftXYGPUbuffer(dx, np.zeros(6, np.float32))
        eng.resetFramePosition()
        eng.loadDriftXYGPUbuffer(np.full(6, 0.25, np.float32), np.zeros(6, np.float32))
        assert not eng.calculateSRRF(raw)
        assert np.isfinite(eng.readSRRFbuffer()).all()
    finally:
        eng.release()
