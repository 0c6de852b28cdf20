"""CPU tests of the oracle: the C restatement against the golden fixtures made by the
reference's own kernels, plus known-answer properties of each stage."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_err


@pytest.mark.parametrize("name", golden_names())
def test_restatement_matches_reference_kernels(oracle_mod, name):
    """The FP32 restatement reproduces the reference kernels' output bit for bit."""
    O = oracle_mod
    g = load_golden(name)
    kw = dict(int_weighting=bool(g["int_weighting"]), drift_x=g.get("drift_x"),
              drift_y=g.get("drift_y"))
    M, fwhm, S = int(g["magnification"]), float(g["fwhm"]), int(g["sensitivity"])
    kind = str(g["kind"])
    if kind == "fht":
        got = O.fht_block(g["interp"], M, fwhm, S, **kw)
    elif kind == "bic":
        got = O.bic_block(g["raw"], M, fwhm, S, mp_correction=bool(g["mp_correction"]), **kw)
    else:
        got = O.block3d(g["raw"], M, fwhm, S, g["theta"], g["shift_x"], g["shift_y"],
                        mp_correction=bool(g["mp_correction"]), **kw)
    np.testing.assert_array_equal(got, g["out"])


@pytest.mark.parametrize("name", golden_names())
def test_fp64_restatement_close_to_reference(oracle_mod, name):
    """FP64 restatement vs the reference's FP32 kernels: within 1e-4 of each slice's range."""
    O = oracle_mod
    g = load_golden(name)
    kw = dict(int_weighting=bool(g["int_weighting"]), drift_x=g.get("drift_x"),
              drift_y=g.get("drift_y"), precision="f64")
    M, fwhm, S = int(g["magnification"]), float(g["fwhm"]), int(g["sensitivity"])
    kind = str(g["kind"])
    if kind == "fht":
        got = O.fht_block(g["interp"], M, fwhm, S, **kw)
    elif kind == "bic":
        got = O.bic_block(g["raw"], M, fwhm, S, mp_correction=bool(g["mp_correction"]), **kw)
    else:
        got = O.block3d(g["raw"], M, fwhm, S, g["theta"], g["shift_x"], g["shift_y"],
                        mp_correction=bool(g["mp_correction"]), **kw)
    ref = g["out"].reshape(4, -1)
    got = got.reshape(4, -1)
    for k in range(4):
        assert rel_err(got[k], ref[k]) < 1e-4, (name, k)


def test_fht_fixture_inputs_reproduce(oracle_mod):
    """The stored interpolated inputs are what the restatement produces from the raw frames."""
    O = oracle_mod
    for name in golden_names("fht"):
        g = load_golden(name)
        np.testing.assert_array_equal(O.fht_interpolate(g["raw"], int(g["magnification"])),
                                      g["interp"])


def test_interpolation_known_answers(oracle_mod):
    O = oracle_mod
    # constant frame stays constant (mean preserving scale), any M
    for M in (2, 3, 5):
        c = np.full((1, 16, 16), 123.0, np.float32)
        np.testing.assert_allclose(O.fht_interpolate(c, M), 123.0, rtol=1e-6)
    # band-limited cosine whose period divides N is reproduced on the fine grid
    N, M = 32, 4
    x = np.arange(N)
    img = (100 + 10 * np.cos(2 * np.pi * 3 * x / N))[None, :].repeat(N, 0)[None].astype(np.float32)
    fine = O.fht_interpolate(img, M)
    xf = (np.arange(N * M)) / M
    expect = 100 + 10 * np.cos(2 * np.pi * 3 * xf / N)
    np.testing.assert_allclose(fine[0, 5], expect, atol=2e-4)
    # phase-0 samples of the fine grid are the raw pixels (power-of-two square input)
    rng = np.random.default_rng(0)
    r = (100 + 20 * rng.random((2, 16, 16))).astype(np.float32)
    np.testing.assert_allclose(O.fht_interpolate(r, 3)[:, ::3, ::3], r, atol=2e-4)
    # unitary-big scale divides the mean by M^2
    np.testing.assert_allclose(O.fht_interpolate(c, 3, scale_mode=1), 123.0 / 9, rtol=1e-6)


def test_interpolation_mirror_padding_non_power_of_two(oracle_mod):
    """Non power-of-two, non-square frames go through mirror padding and a centred crop; a
    constant frame and a linear ramp's mean survive it."""
    O = oracle_mod
    c = np.full((1, 12, 20), 50.0, np.float32)
    out = O.fht_interpolate(c, 3)
    assert out.shape == (1, 36, 60)
    np.testing.assert_allclose(out, 50.0, rtol=1e-5)


def test_constant_frames_give_zero_rgc(oracle_mod):
    """A constant frame has zero gradient: CGLH = 0, so AVG = VAR = TAC2 = 0, INT = constant."""
    O = oracle_mod
    c = np.full((4, 24, 24), 77.0, np.float32)
    out = O.fht_block(c, 2, 1.5, 1)
    np.testing.assert_allclose(out[:3], 0.0, atol=1e-6)
    np.testing.assert_allclose(out[3], 77.0, rtol=1e-6)
    ref = O.ref_fht_block(c, 2, 1.5, 1) if O.ref_available() else out
    np.testing.assert_array_equal(out, ref)


def test_radial_spot_peaks_at_centre(oracle_mod):
    """A radially symmetric spot gives its CGLH maximum at the spot centre, and the map is
    symmetric under x <-> y (the Roberts-cross staggering is the same along both axes)."""
    O = oracle_mod
    n = 32
    yy, xx = np.mgrid[0:n, 0:n] + 0.5
    spot = 100 + 500 * np.exp(-((xx - 16) ** 2 + (yy - 16) ** 2) / (2 * 2.0 ** 2))
    out = O.fht_block(spot[None].astype(np.float32), 1, 2.0, 1, int_weighting=False)
    avg = out[0]
    iy, ix = np.unravel_index(np.argmax(avg), avg.shape)
    assert abs(iy - 15.5) <= 1 and abs(ix - 15.5) <= 1
    np.testing.assert_allclose(avg, avg.T, atol=1e-5)


def test_var_of_constant_sequence_is_zero(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(3)
    f = (100 + 50 * rng.random((1, 24, 24))).astype(np.float32)
    stack = np.repeat(f, 5, axis=0)
    out = O.fht_block(stack, 2, 1.5, 1, precision="f64")
    assert np.abs(out[1]).max() < 1e-6 * max(1.0, np.abs(out[0]).max() ** 2)
    # TAC2 of a constant sequence equals E[X^2] - E[X]^2 = 0 as well
    assert np.abs(out[2]).max() < 1e-6 * max(1.0, np.abs(out[0]).max() ** 2)


def test_mfm_reshape(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(5)
    frames = rng.random((2, 30, 36)).astype(np.float32) * 100
    roi = np.array([4, 0, 8], np.float32)
    coeff = np.array([1.0, 2.0, 0.5], np.float32)
    planes = O.mfm_reshape(frames, 3, roi, coeff, 10.0)
    assert planes.shape == (2, 3, 10, 12)
    np.testing.assert_allclose(planes[:, 0], (frames[:, 10:20, 12:24] - 10) / 1.0, rtol=1e-6)
    np.testing.assert_allclose(planes[:, 1], (frames[:, 0:10, 0:12] - 10) / 2.0, rtol=1e-6)
    np.testing.assert_allclose(planes[:, 2], (frames[:, 20:30, 24:36] - 10) / 0.5, rtol=1e-6)
