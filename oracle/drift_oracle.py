"""TEST INFRASTRUCTURE ONLY -- float64 restatement of frame drift estimation,
XYShiftCalculator.calculateShiftArray (XYShiftCalculator.java:26-48), the checker for
esrrf_estimate_drift.

The reference builds NanoJ-Core's cross-correlation map of each frame against the block's first
frame (CrossCorrelationMap.calculateCrossCorrelationMap) and takes the sub-pixel position of its
peak (EstimateShiftAndTilt.getShiftFromCrossCorrelationPeak, MAX_FITTING), negated
(XYShiftCalculator.java:42-44).  NanoJ-Core is not in the reference tree, so this module restates
the published method rather than that library's code, and parity with NanoJ-Core's own numbers is
unpinned:
  C_f(s) = sum_p (ref(p) - mean ref) frame_f((p + s) mod size)     (numpy FFT, float64)
over the lags |sx|, |sy| <= R, the first arg-max in row-major order, and the stationary point of the
least-squares quadratic through the 3 x 3 samples around it (clamped to +-1).  The shift is the
displacement d of the frame's content (frame(p) = ref(p - d)), which is what liveSRRF.cl:263 adds to
the sampling position.  Only tests/ use this module.
"""
from __future__ import annotations

import numpy as np


def window(width, height, max_shift=None):
    lim = (min(width, height) - 1) // 2
    R = max_shift if max_shift and max_shift > 0 else 31
    return max(1, min(R, lim))


def ccm(frames, ref_frame=0, R=None):
    """[T][2R+1][2R+1] float64 maps, lag (sy, sx) at [sy + R][sx + R]."""
    f = np.asarray(frames, np.float64)
    if f.ndim == 2:
        f = f[None]
    T, H, W = f.shape
    R = window(W, H) if R is None else R
    r = f[ref_frame] - f[ref_frame].mean()
    Fr = np.conj(np.fft.fft2(r))
    full = np.real(np.fft.ifft2(Fr[None] * np.fft.fft2(f), axes=(-2, -1)))  # full[t, sy mod H, sx mod W]
    lags = np.arange(-R, R + 1)
    return full[:, (lags % H)[:, None], (lags % W)[None, :]]


def ccm_direct(frames, ref_frame, R):
    """The same map by explicit sums (small sizes only): pins the FFT form."""
    f = np.asarray(frames, np.float64)
    T, H, W = f.shape
    r = f[ref_frame] - f[ref_frame].mean()
    out = np.zeros((T, 2 * R + 1, 2 * R + 1))
    for sy in range(-R, R + 1):
        for sx in range(-R, R + 1):
            g = np.roll(f, (-sy, -sx), axis=(1, 2))  # g[p] = f[p + s]
            out[:, sy + R, sx + R] = (r[None] * g).sum(axis=(1, 2))
    return out


def quadratic_peak(v):
    """Stationary point of the least-squares quadratic through v[3][3] (x, y in -1..1), clamped."""
    v = np.asarray(v, np.float64)
    x = np.array([-1.0, 0.0, 1.0])
    X, Y = np.meshgrid(x, x)
    S, Sx, Sy = v.sum(), (X * v).sum(), (Y * v).sum()
    Sxy, Sxx, Syy = (X * Y * v).sum(), (X * X * v).sum(), (Y * Y * v).sum()
    b, c, e = Sx / 6.0, Sy / 6.0, Sxy / 4.0
    d, f = Sxx / 2.0 - S / 3.0, Syy / 2.0 - S / 3.0
    det = 4.0 * d * f - e * e
    ox = oy = 0.0
    if det != 0.0:
        ox = (-2.0 * f * b + e * c) / det
        oy = (-2.0 * d * c + e * b) / det
    return float(np.clip(ox, -1, 1)), float(np.clip(oy, -1, 1))


def peaks(maps, R):
    side = 2 * R + 1
    sx = np.empty(len(maps))
    sy = np.empty(len(maps))
    for t, m in enumerate(maps):
        b = int(np.argmax(m))
        py, px = divmod(b, side)
        ox = oy = 0.0
        if 0 < px < side - 1 and 0 < py < side - 1:
            ox, oy = quadratic_peak(m[py - 1:py + 2, px - 1:px + 2])
        sx[t] = px - R + ox
        sy[t] = py - R + oy
    return sx, sy


def estimate_drift(frames, ref_frame=0, max_shift=None):
    f = np.asarray(frames)
    R = window(f.shape[-1], f.shape[-2], max_shift)
    return peaks(ccm(f, ref_frame, R), R)


def shifted_stack(seed, T, H, W, shifts, n_spots=40, sigma=2.0):
    """Frames of Gaussian spots whose content is displaced by shifts[t] = (dx, dy) pixels: each spot
    is drawn at its position plus the shift, so frame_t(p) = frame_0(p - d_t) up to the edges."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform([0.15 * W, 0.15 * H], [0.85 * W, 0.85 * H], size=(n_spots, 2))
    amp = rng.uniform(200, 1000, n_spots)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    out = np.empty((T, H, W))
    for t in range(T):
        dx, dy = shifts[t]
        img = np.full((H, W), 100.0)
        for (px, py), a in zip(pos, amp):
            img += a * np.exp(-((xx - px - dx) ** 2 + (yy - py - dy) ** 2) / (2 * sigma * sigma))
        out[t] = img
    return out
