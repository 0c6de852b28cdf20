"""GPU tests of esrrf_estimate_drift (restatement of XYShiftCalculator.calculateShiftArray,
XYShiftCalculator.java:26-48) against the float64 oracle (oracle/drift_oracle.py).

Maps: within 1e-6 of each map's largest magnitude (each 32-pixel row of products summed in FP32,
rows in FP64; an emulation of that order gives 1.4e-7 on the first case).  Shifts: within 1e-3 px of the oracle's (the quadratic fit reads differences of neighbouring
map values).  Cases: uint16 and float32 frames, sizes that are not multiples of the tiles, a window
clamped by a small frame, a window of several lag tiles, a reference frame other than the first.
The mirror class and the shifts' use by the engine (loadDriftXYGPUbuffer) are covered end to end."""
import numpy as np
import pytest

from conftest import rel_err
from oracle import drift_oracle as D

pytestmark = pytest.mark.gpu

CASES = [
    # w, h, T, max_shift, ref, u16
    (96, 80, 6, None, 0, True),
    (131, 77, 5, None, 2, False),
    (20, 17, 4, None, 0, True),     # R clamped to 8
    (200, 180, 3, 80, 1, False),    # 161 x 161 lags: three lag tiles a side
    (512, 512, 4, None, 0, True),
]


def stack(w, h, T, seed):
    rng = np.random.default_rng(seed)
    shifts = [(0.0, 0.0)] + [tuple(rng.uniform(-3, 3, 2)) for _ in range(T - 1)]
    return D.shifted_stack(seed, T, h, w, shifts, n_spots=max(6, w * h // 400)), shifts


@pytest.mark.parametrize("w,h,T,ms,ref,u16", CASES)
def test_drift_matches_oracle(esrrf_mod, w, h, T, ms, ref, u16):
    f, _ = stack(w, h, T, w + h)
    f = np.round(f).astype(np.uint16) if u16 else f.astype(np.float32)
    R = D.window(w, h, ms)
    assert esrrf_mod.drift_window(w, h, ms) == R
    sx, sy, maps = esrrf_mod.estimate_drift(f, ref, ms, return_map=True)
    want = D.ccm(f.astype(np.float64), ref, R)
    assert maps.shape == want.shape
    for t in range(T):
        err = np.abs(maps[t] - want[t]).max() / np.abs(want[t]).max()
        assert err < 1e-6, (t, err)
    ox, oy = D.peaks(want, R)
    np.testing.assert_allclose(sx, ox, atol=1e-3)
    np.testing.assert_allclose(sy, oy, atol=1e-3)


def test_known_subpixel_shifts(esrrf_mod):
    shifts = [(0, 0), (0.3, -0.2), (-1.45, 0.7), (2.5, 2.25), (-4.1, -3.6), (6.2, -5.9)]
    f = D.shifted_stack(7, len(shifts), 128, 128, shifts).astype(np.float32)
    sx, sy = esrrf_mod.estimate_drift(f)
    np.testing.assert_allclose(sx, [s[0] for s in shifts], atol=0.05)
    np.testing.assert_allclose(sy, [s[1] for s in shifts], atol=0.05)


def test_integer_roll_is_exact(esrrf_mod):
    base = np.round(D.shifted_stack(1, 1, 64, 80, [(0, 0)])[0]).astype(np.uint16)
    moved = [np.roll(base, (dy, dx), axis=(0, 1)) for dx, dy in [(0, 0), (3, -2), (-7, 5), (11, 11)]]
    sx, sy = esrrf_mod.estimate_drift(np.stack(moved))
    np.testing.assert_allclose(sx, [0, 3, -7, 11], atol=1e-4)
    np.testing.assert_allclose(sy, [0, -2, 5, 11], atol=1e-4)


def test_xyshiftcalculator_mirror(esrrf_mod):
    f, shifts = stack(64, 64, 8, 11)
    calc = esrrf_mod.XYShiftCalculator(f.astype(np.float32))
    calc.calculateShiftArray(3, 5)  # 1-based: frames 2..6, reference frame 2
    sx, sy = D.estimate_drift(f[2:7])
    np.testing.assert_allclose(calc.shiftX, sx, atol=1e-3)
    np.testing.assert_allclose(calc.shiftY, sy, atol=1e-3)
    with pytest.raises(esrrf_mod.EsrrfError):
        calc.calculateShiftArray(6, 5)


def test_estimated_drift_drives_the_engine(esrrf_mod, oracle_mod):
    """Shifts estimated on the GPU, loaded with loadDriftXYGPUbuffer, give the oracle's
    drift-corrected block for the same shifts; and the correction re-aligns a drifting stack.

    The stack carries camera noise (sigma 10 ADU): on noise-free spots over a flat background the
    gradient directions in the flat regions come from rounding alone, and a 2e-7 perturbation of
    the interpolated frames moves the VAR slice by 1e-2 of its range in the oracle itself."""
    f, shifts = stack(48, 40, 6, 5)
    f = f + np.random.default_rng(1).normal(0, 10, f.shape)
    raw = np.round(np.clip(f, 0, None)).astype(np.uint16)
    sx, sy = esrrf_mod.estimate_drift(raw)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(48, 40, 2, 1.5, 2, 6, 6)
    try:
        eng.loadDriftXYGPUbuffer(sx, sy)
        eng.resetFramePosition()
        assert not eng.calculateSRRF(raw)
        got = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw.astype(np.float32), 2), 2, 1.5, 2,
                               drift_x=sx, drift_y=sy)
    for k in range(4):
        assert rel_err(got[k], ref[k]) < 1e-4, k
    np.testing.assert_allclose(sx, [s[0] for s in shifts], atol=0.1)
    np.testing.assert_allclose(sy, [s[1] for s in shifts], atol=0.1)


def test_bad_arguments(esrrf_mod):
    f = np.zeros((2, 16, 16), np.float32)
    with pytest.raises(esrrf_mod.EsrrfError):
        esrrf_mod.estimate_drift(f, ref_frame=2)
    with pytest.raises(esrrf_mod.EsrrfError):
        esrrf_mod.estimate_drift(np.zeros((2, 2, 16), np.float32))
