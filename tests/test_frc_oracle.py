"""CPU checks of the FRC oracle (oracle/frc_oracle.py, the checker for esrrf_frc; the sweep's FRC
resolution, gui/ParametersSweep_.java:403-447): the FFT ring sums against an explicit DFT, exact
integer ring rounding, the window, the crossing rule and the ordering of resolutions."""
import math

import numpy as np
import pytest

from oracle import frc_oracle as F


def test_padded_size_and_rings():
    assert F.padded_size(10, 7) == 32 and F.padded_size(100, 80) == 128 and F.padded_size(129, 3) == 256
    r = F.rings(64)
    f = np.fft.fftfreq(64, 1 / 64)
    want = np.array([[int(math.floor(math.hypot(u, v) + 0.5)) for v in f] for u in f])
    np.testing.assert_array_equal(r, want)


def test_tukey_window():
    w = F.tukey(33)
    assert w[0] == 0.0 and w[-1] == 0.0 and w[16] == 1.0
    np.testing.assert_allclose(w, w[::-1])
    # tapers over the outer eighth: a = (n - 1) / 8 = 4 samples
    assert np.all(np.diff(w[:5]) > 0) and np.all(w[4:29] == 1.0)


def test_ring_sums_match_explicit_dft():
    rng = np.random.default_rng(2)
    a, b = rng.normal(size=(20, 27)), rng.normal(size=(20, 27))
    frc, N = F.curve(a, b)
    win = F.tukey(20)[:, None] * F.tukey(27)[None, :]
    pa = np.zeros((N, N)); pb = np.zeros((N, N))
    pa[:20, :27] = (a - a.mean()) * win
    pb[:20, :27] = (b - b.mean()) * win
    k = np.arange(N)
    D = np.exp(-2j * np.pi * np.outer(k, k) / N)  # explicit DFT matrix
    Fa, Fb = D @ pa @ D.T, D @ pb @ D.T
    r = F.rings(N)
    for ring in (1, 5, 16):
        m = r == ring
        c = np.real(Fa[m] * np.conj(Fb[m])).sum()
        want = c / np.sqrt((np.abs(Fa[m]) ** 2).sum() * (np.abs(Fb[m]) ** 2).sum())
        assert abs(frc[ring] - want) < 1e-10


def test_identical_and_independent_images():
    a, _ = F.split_images(1, 100, 80, 0.1, 0.0)
    frc, _ = F.curve(a, a)
    np.testing.assert_allclose(frc[1:], 1.0, atol=1e-12)
    assert math.isnan(F.fire(a, a)[0])            # never drops below 1/7
    # independent noise: the curve is at 1/7 within a few rings (rings 1-2 hold 8-12 frequencies,
    # so their correlation is itself noisy): NaN or a resolution of more than a third of N
    rng = np.random.default_rng(0)
    for _ in range(5):
        r = F.fire(rng.normal(size=(64, 64)), rng.normal(size=(64, 64)))[0]
        assert math.isnan(r) or r > 64 / 3


def test_resolution_orders_with_band_limit_and_noise():
    res = [F.fire(*F.split_images(1, 128, 128, c, 5.0))[0] for c in (0.05, 0.1, 0.2)]
    assert res[0] > res[1] > res[2] > 2.0
    noisy = F.fire(*F.split_images(1, 128, 128, 0.1, 40.0))[0]
    assert noisy > res[1]
    # pixel size scales the result
    a, b = F.split_images(1, 128, 128, 0.1, 5.0)
    assert F.fire(a, b, pixel_size=0.025)[0] == pytest.approx(res[1] * 0.025)


def test_crossing_interpolation():
    # a curve crossing 1/7 between rings 3 and 4 -> q = 3 + (c3 - 1/7) / (c3 - c4)
    c3, c4 = 0.5, 0.1
    q = 3 + (c3 - 1 / 7) / (c3 - c4)
    assert 3 < q < 4
