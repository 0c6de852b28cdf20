"""GPU parity at the benchmarked configurations, against the reference's own kernels.

The checker is ``oracle/_ref`` (liveSRRF_noInterpolation.cl compiled for the host and replayed in
LiveSRRF_CL.java's launch order) where it was built, else the C restatement that is bit-identical
to it on every golden fixture.  The interpolated frames the checker reads come from the float64
FFT form of FourierInterpolation.java's map.

* 512 x 512 uint16 frames at M4, radius 1.5, sensitivity 2 (the headline workload's frame size
  and parameters): a 4-frame block cut into launches of 2 frames, so that a launch edge falls
  inside the block and TAC2 pairs across it.
* The parameter sweep's per-frame CGLH mode at M2 and M4 with radii 0.5 and 3.0 (at M4 radius 3.0
  has a 26-wide tap box, the largest of the sweep workload) on a 64 x 64 crop, uneven blocks.
* The fidelity-loss adjoint at M4 (the 256 x 256 x 100 workload's magnification, 18-wide tap box)
  on a 48 x 48 x 8 stack: radius, sensitivity, re-blur sigma and pixel gradients against central
  finite differences (h = 1e-3) of the float64 loss.
* The bicubic path on 512 x 512 uint16 frames at M4, radius 1.5, S2 with MP correction (the bicubic
  workload), 3 frames in launches of 2, against liveSRRF.cl compiled for the host.
* The 3-D path on 9 planes of 128 x 128 at M3, radius 1.5, S1 with per-plane alignment and MP
  correction (the 3-D workload's planes, calibration and parameters), 3 timepoints in launches of 2,
  against live3DSRRF.cl compiled for the host.
* 1024 x 1024 frames at M4 (4096 x 4096 output), the largest tested, against the reference kernels.

Tolerance: each slice within 1e-4 of its dynamic range; gradients within 1e-3 relative (pixel
gradients with a floor at 20 % of the largest one checked).
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _ref_block(O, interp, M, fwhm, S, frames_per_load=0):
    if O.ref_available():
        return O.ref_fht_block(interp, M, fwhm, S, frames_per_load=frames_per_load)
    return O.fht_block(interp, M, fwhm, S)


def test_headline_frame_size_against_reference_kernels(esrrf_mod, oracle_mod):
    from esrrf import synth
    raw = synth.make_stack("fht512", frames=4)
    assert raw.dtype == np.uint16 and raw.shape == (4, 512, 512)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(512, 512, 4, 1.5, 2, 4, 4, framesPerLaunch=2)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(raw)
        got = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    interp = oracle_mod.fht_interpolate_fft(raw.astype(np.float32), 4)
    ref = _ref_block(oracle_mod, interp, 4, 1.5, 2, frames_per_load=2)
    assert np.abs(ref[2]).max() > 0
    for k in range(4):
        e = rel_err(got[k], ref[k])
        assert e < TOL, f"slice {k}: {e:.3g} of range"


def test_sweep_cglh_mode_large_and_small_radii(esrrf_mod, oracle_mod):
    from esrrf import synth
    raw = synth.small_stack(61, 12, 64, 64, emitters=40)
    mags, radii, sens = [2, 4], [0.5, 3.0], [1, 4]
    blocks = [(0, 5), (5, 7), (2, 9)]
    sw = esrrf_mod.Sweep(64, 64, 12, mags, radii, sens, blocks)
    try:
        res = sw.run(raw)
    finally:
        sw.release()
    assert len(res) == len(mags) * len(radii) * len(sens) * len(blocks)
    interp = {M: oracle_mod.fht_interpolate(raw.astype(np.float32), M) for M in mags}
    for (M, r, S, (st, ln)), got in res.items():
        ref = _ref_block(oracle_mod, interp[M][st:st + ln], M, r, S)
        for k in range(4):
            e = rel_err(got[k], ref[k])
            assert e < TOL, (M, r, S, st, ln, k, e)


def test_adjoint_at_m4_against_finite_differences(esrrf_mod):
    from esrrf import synth
    from oracle import adjoint_oracle as A
    raw = synth.small_stack(72, 8, 48, 48, emitters=20).astype(np.float32)
    M, fwhm, S, sig = 4, 1.5, 2.0, 1.3
    pix = [(0, 5, 5), (3, 20, 30), (7, 47, 0), (5, 24, 24)]
    fd = A.fd_gradient(raw, M, fwhm, S, sig, pixels=pix)
    L64 = A.loss(raw, M, fwhm, S, sig)
    adj = esrrf_mod.Adjoint(48, 48, 8, M)
    try:
        L, g, gf = adj.loss_and_grad(raw, fwhm, S, sig)
        gf = gf.cpu().numpy()
    finally:
        adj.release()
    assert abs(L - L64) <= 1e-4 * abs(L64), (L, L64)
    for k in ("fwhm", "S", "sigma"):
        assert abs(g[k] - fd[k]) <= 1e-3 * abs(fd[k]), (k, g[k], fd[k])
    # pixel gradients: 1e-3 relative, with a floor of 1e-3 x 20 % of the largest one checked (the
    # FP32 forward pass leaves ~1e-7 of absolute noise on the smallest components at this size)
    scale = max(abs(v) for v in fd["pixels"].values())
    for (t, y, x), v in fd["pixels"].items():
        assert abs(gf[t, y, x] - v) <= 1e-3 * max(abs(v), 0.2 * scale), ((t, y, x), gf[t, y, x], v)


def test_bicubic_headline_frame_size_against_reference_kernels(esrrf_mod, oracle_mod):
    from esrrf import synth
    from test_gpu_bic3d import assert_close, run
    raw = synth.make_stack("fht512", frames=3)
    got, _ = run(esrrf_mod, raw, 4, 1.5, 2, mp=True, fht=False, frames_per_launch=2)
    if oracle_mod.ref_available():
        ref = oracle_mod.ref_bic_block(raw, 4, 1.5, 2, mp_correction=True, frames_per_load=2)
    else:
        ref = oracle_mod.bic_block(raw.astype(np.float32), 4, 1.5, 2, mp_correction=True)
    assert np.abs(ref[2]).max() > 0
    assert_close(got, ref, "bicubic 512x512 M4")


def test_3d_workload_size_against_reference_kernels(esrrf_mod, oracle_mod):
    from esrrf import synth
    from test_gpu_bic3d import assert_close, calib, run, tile_planes
    planes = synth.make_stack("mfm3d", frames=3)
    n, P, h, w = planes.shape
    assert (P, h, w) == (9, 128, 128)
    roi = np.array([4, 0, 1, 2, 3, 5, 6, 7, 8], np.float32)
    theta = np.linspace(-0.5, 0.5, P).astype(np.float32)
    sx = np.linspace(-0.2, 0.2, P).astype(np.float32)
    sy = np.linspace(0.1, -0.1, P).astype(np.float32)
    got, _ = run(esrrf_mod, tile_planes(planes.astype(np.float32), roi), 3, 1.5, 1, mp=True,
                 calib=calib(P, theta, sx, sy, roi), frames_per_launch=2)
    if oracle_mod.ref_available():
        ref = oracle_mod.ref_3d_block(planes, 3, 1.5, 1, theta, sx, sy, mp_correction=True,
                                      frames_per_load=2)
    else:
        ref = oracle_mod.block3d(planes.astype(np.float32), 3, 1.5, 1, theta, sx, sy, mp_correction=True)
    assert got.shape == (4 * P * 3, h * 3, w * 3)
    assert_close(got, ref, "3-D 9 x 128 x 128 M3")


def test_large_frames_against_reference_kernels(esrrf_mod, oracle_mod):
    """1024 x 1024 uint16 frames at M4 (padded size 1024, 4096 x 4096 output): the largest frames
    of these tests, through the tensor-core interpolation and the fused kernel (2 frames in one
    launch), against the reference kernels on the float64 FFT interpolation."""
    from esrrf import synth
    wl = synth.Workload("big", 1024, 1024, 2, 4, 1.5, 2, emitters=4000, filaments=30, seed=77)
    raw = synth.make_stack(wl)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(1024, 1024, 4, 1.5, 2, 2, 2)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(raw)
        got = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    interp = oracle_mod.fht_interpolate_fft(raw.astype(np.float32), 4)
    assert rel_err(got[3], interp.mean(axis=0)) < 2e-6
    ref = _ref_block(oracle_mod, interp, 4, 1.5, 2)
    for k in range(4):
        e = rel_err(got[k], ref[k])
        assert e < TOL, f"slice {k}: {e:.3g} of range"
