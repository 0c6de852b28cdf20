"""CPU checks of the drift-estimation oracle (restatement of XYShiftCalculator.calculateShiftArray,
XYShiftCalculator.java:26-48): the FFT map against explicit sums, integer shifts recovered exactly,
sub-pixel shifts of drawn spots within 0.05 px, the sign convention and the lag window."""
import numpy as np
import pytest

from oracle import drift_oracle as D


def test_fft_map_matches_direct_sums():
    rng = np.random.default_rng(3)
    f = rng.uniform(0, 1000, (3, 13, 17))
    R = 5
    np.testing.assert_allclose(D.ccm(f, 1, R), D.ccm_direct(f, 1, R), rtol=0, atol=1e-8 * np.abs(D.ccm_direct(f, 1, R)).max())


@pytest.mark.parametrize("d", [(0, 0), (3, -2), (-7, 5), (11, 11)])
def test_integer_shift_exact(d):
    base = D.shifted_stack(1, 1, 64, 80, [(0, 0)])[0]
    moved = np.roll(base, (d[1], d[0]), axis=(0, 1))  # content displaced by +d
    sx, sy = D.estimate_drift(np.stack([base, moved]))
    assert abs(sx[0]) < 1e-9 and abs(sy[0]) < 1e-9
    assert abs(sx[1] - d[0]) < 1e-9 and abs(sy[1] - d[1]) < 1e-9


def test_subpixel_shifts():
    shifts = [(0, 0), (0.3, -0.2), (-1.45, 0.7), (2.5, 2.25), (-4.1, -3.6)]
    f = D.shifted_stack(7, len(shifts), 96, 96, shifts)
    sx, sy = D.estimate_drift(f)
    for t, (dx, dy) in enumerate(shifts):
        assert abs(sx[t] - dx) < 0.05 and abs(sy[t] - dy) < 0.05, (t, sx[t], sy[t], dx, dy)


def test_reference_frame_and_window():
    shifts = [(1.0, 2.0), (0.0, 0.0), (-2.0, 1.0)]
    f = D.shifted_stack(9, 3, 64, 64, shifts)
    sx, sy = D.estimate_drift(f, ref_frame=1)
    np.testing.assert_allclose(sx, [1.0, 0.0, -2.0], atol=0.05)
    np.testing.assert_allclose(sy, [2.0, 0.0, 1.0], atol=0.05)
    assert D.window(512, 512) == 31
    assert D.window(20, 17) == 8
    assert D.window(200, 180, 80) == 80
    assert D.window(200, 180, 500) == 89


def test_quadratic_peak_recovers_paraboloid_vertex():
    x = np.array([-1.0, 0.0, 1.0])
    X, Y = np.meshgrid(x, x)
    v = 5 - (X - 0.3) ** 2 - 2 * (Y + 0.4) ** 2 + 0.2 * (X - 0.3) * (Y + 0.4)
    ox, oy = D.quadratic_peak(v)
    assert abs(ox - 0.3) < 1e-12 and abs(oy + 0.4) < 1e-12
