"""GPU tests of the tensor-core (tcgen05, three-term TF32) form of the Fourier interpolation's two
dense passes against the FP32 SIMT kernels (ESRRF_INTERP_GEMM=simt) and the float64
interpolation (FourierInterpolation.java's map by numpy FFT).

The INT slice of a block is the frame average of the interpolated frames, so it exposes the
interpolation directly.  Sizes cover partial tiles in both directions (output rows not a multiple
of 128, columns not a multiple of 256), wide mirror padding and a 512 x 512 frame; padded sizes
below 128 must take the SIMT kernels.  Tolerance: within 2e-6 of the slice's dynamic range of the float64
interpolation, and no worse than twice the SIMT kernels' error plus 1e-6 of range.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def run_block(esrrf, frames, M, fwhm=1.5, S=2):
    eng = esrrf.LiveSRRF_CL()
    n = frames.shape[0]
    eng.initialise(frames.shape[-1], frames.shape[-2], M, fwhm, S, n, n)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(frames)
        return eng.readSRRFbuffer().copy()
    finally:
        eng.release()


CASES = [
    (96, 160, 5, 2),   # N 256, 480 x 800 output
    (512, 512, 4, 2),  # N 512
    (200, 136, 3, 2),  # N 256, 600 x 408 output: partial tiles in both directions
    (130, 100, 2, 2),  # N 256 with wide mirror padding, 260 x 200 output: a 4-column last tile
]
# padded sizes below 128 run the SIMT kernels (a 128-row tile would be mostly padding)
SMALL = [(40, 24, 3, 3), (20, 32, 2, 2)]


def both_paths(esrrf, monkeypatch, raw, M):
    monkeypatch.delenv("ESRRF_INTERP_GEMM", raising=False)
    tc = run_block(esrrf, raw, M)
    monkeypatch.setenv("ESRRF_INTERP_GEMM", "simt")
    simt = run_block(esrrf, raw, M)
    return tc, simt


@pytest.mark.parametrize("w,h,M,T", CASES)
def test_tc_interpolation_matches_fp64(esrrf_mod, monkeypatch, w, h, M, T):
    from esrrf import synth
    from oracle import adjoint_oracle as A
    raw = synth.small_stack(100 + w + h + M, T, h, w).astype(np.float32)
    ref = A.interpolate_f64(raw, M).mean(axis=0)
    tc, simt = both_paths(esrrf_mod, monkeypatch, raw, M)
    e_tc, e_simt = rel_err(tc[3], ref), rel_err(simt[3], ref)
    # different rounding shows that the tensor-core passes ran
    assert not np.array_equal(tc[3], simt[3])
    assert e_tc < 2e-6 and e_tc <= 2 * e_simt + 1e-6, (e_tc, e_simt)
    # the remaining slices agree with the SIMT path's to the engine's parity bar
    for k in range(3):
        assert rel_err(tc[k], simt[k]) < 1e-4, (k, rel_err(tc[k], simt[k]))


@pytest.mark.parametrize("w,h,M,T", SMALL)
def test_small_frames_use_simt(esrrf_mod, monkeypatch, w, h, M, T):
    from esrrf import synth
    from oracle import adjoint_oracle as A
    raw = synth.small_stack(100 + w + h + M, T, h, w).astype(np.float32)
    ref = A.interpolate_f64(raw, M).mean(axis=0)
    tc, simt = both_paths(esrrf_mod, monkeypatch, raw, M)
    np.testing.assert_array_equal(tc, simt)
    assert rel_err(tc[3], ref) < 2e-6


def test_tc_interpolation_u16_and_chunks(esrrf_mod, oracle_mod, monkeypatch):
    """uint16 input pushed in uneven GPU loads through the tensor-core passes."""
    from esrrf import synth
    monkeypatch.delenv("ESRRF_INTERP_GEMM", raising=False)
    raw = synth.small_stack(5, 9, 128, 128)
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw.astype(np.float32), 2), 2, 1.5, 2)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(128, 128, 2, 1.5, 2, 9, 9, framesPerLaunch=4)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(raw[:2])
        assert not eng.calculateSRRF(raw[2:])
        got = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    for k in range(4):
        assert rel_err(got[k], ref[k]) < 1e-4, k
