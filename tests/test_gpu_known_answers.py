"""Known-answer checks of the GPU path itself, beside the oracle parity tests: a band-limited
cosine whose period divides the frame size comes out of the Fourier interpolation (tensor-core and
SIMT forms) exactly on the fine grid; a radially symmetric spot gives its RGC maximum at the spot
centre and a map symmetric under x <-> y around it; TAC2 of independent frames averages to ~0 while their
VAR does not; a constant stack gives zero convergence on every path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def block(esrrf, frames, M, fwhm=1.5, S=1, intw=True):
    eng = esrrf.LiveSRRF_CL()
    n = frames.shape[0]
    eng.initialise(frames.shape[-1], frames.shape[-2], M, fwhm, S, n, n, intWeighting=intw)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(frames)
        return eng.readSRRFbuffer().copy()
    finally:
        eng.release()


@pytest.mark.parametrize("N,M,k", [(256, 4, 5), (32, 4, 3), (128, 3, 7)])
def test_band_limited_cosine_is_reproduced(esrrf_mod, N, M, k):
    x = np.arange(N)
    row = 100 + 10 * np.cos(2 * np.pi * k * x / N)
    frames = np.repeat(row[None, None, :], N, axis=1).repeat(2, axis=0).astype(np.float32)
    out = block(esrrf_mod, frames, M)
    xf = np.arange(N * M) / M
    expect = 100 + 10 * np.cos(2 * np.pi * k * xf / N)
    interp = out[3]  # INT: the frame average of the interpolated frames
    np.testing.assert_allclose(interp[N * M // 2], expect, atol=2e-4)
    np.testing.assert_allclose(interp[::7].std(axis=0), 0.0, atol=1e-3)  # constant along y (1e-4 of the amplitude)


def test_radial_spot_peaks_at_centre(esrrf_mod):
    n, M = 32, 2
    yy, xx = np.mgrid[0:n, 0:n] + 0.5
    spot = 100 + 500 * np.exp(-((xx - 16) ** 2 + (yy - 16) ** 2) / (2 * 2.0 ** 2))
    out = block(esrrf_mod, np.repeat(spot[None], 2, axis=0).astype(np.float32), M, fwhm=2.0, intw=False)
    avg = out[0]
    iy, ix = np.unravel_index(np.argmax(avg), avg.shape)
    c = 16 * M - 0.5  # the spot centre on the fine grid
    assert abs(iy - c) <= 1.5 and abs(ix - c) <= 1.5, (iy, ix)
    # symmetric where the spot has gradients (within 3 sigma); on the flat, noise-free background
    # the gradient directions come from rounding alone and the map there is noise
    win = avg[int(c) - 11:int(c) + 13, int(c) - 11:int(c) + 13]
    np.testing.assert_allclose(win, win.T, atol=1e-4 * (avg.max() - avg.min()))


def test_tac2_of_independent_frames_is_small(esrrf_mod):
    rng = np.random.default_rng(11)
    frames = rng.poisson(200.0, size=(200, 64, 64)).astype(np.float32)
    out = block(esrrf_mod, frames, 2)
    var, tac2 = out[1][8:-8, 8:-8], out[2][8:-8, 8:-8]
    assert var.mean() > 0
    assert abs(tac2.mean()) < 0.05 * var.mean(), (tac2.mean(), var.mean())


def test_constant_frames_give_zero_convergence(esrrf_mod):
    """A constant stack has a zero gradient everywhere, so no tap is inward: CGLH = 0, hence AVG,
    VAR and TAC2 are 0, and INT is the constant -- on the FHT path (a frame that needs mirror
    padding: the interpolation of a constant is the constant), the bicubic path with and without
    MP correction, and the 3-D path."""
    from test_gpu_bic3d import calib, run, tile_planes
    c = 123.0
    frames = np.full((5, 48, 64), c, np.float32)
    fht = block(esrrf_mod, frames, 4, 1.5, 2)
    assert np.abs(fht[:3]).max() == 0.0
    np.testing.assert_allclose(fht[3], c, rtol=1e-6)
    for mp in (False, True):
        bic, _ = run(esrrf_mod, frames, 3, 1.5, 1, mp=mp, fht=False)
        assert np.abs(bic[:3]).max() == 0.0, mp
        np.testing.assert_allclose(bic[3], c, rtol=1e-5)
    P = 5
    planes = np.full((4, P, 24, 20), c, np.float32)
    roi = np.array([4, 0, 8, 5, 1], np.float32)
    zeros = np.zeros(P, np.float32)
    v3d, _ = run(esrrf_mod, tile_planes(planes, roi), 3, 1.5, 1, mp=False, calib=calib(P, zeros, zeros, zeros, roi))
    v3d = v3d.reshape(4, -1)
    assert np.abs(v3d[:3]).max() == 0.0
    np.testing.assert_allclose(v3d[3], c, rtol=1e-5)
