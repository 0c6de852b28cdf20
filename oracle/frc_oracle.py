"""TEST INFRASTRUCTURE ONLY -- float64 restatement of the Fourier ring correlation / FIRE number
the parameter sweep reports (gui/ParametersSweep_.java:403-447: FRC.calculateFireNumber(odd,
even, FIXED_1_OVER_7) x the reconstruction's pixel size), the checker for esrrf_frc.

NanoJ-Core's FRC class is not in the reference tree, so this restates the published method
(Nieuwenhuizen et al., Nat. Methods 10:557, 2013) with the choices esrrf_frc documents, and parity
with NanoJ-Core's numbers is unpinned: mean-subtracted images times a Tukey window (cosine tapers
over the outer eighth of each axis), zero-padded at the origin to N x N (N the next power of two
>= max(width, height, 32)); FRC(r) = sum Re(F1 conj F2) / sqrt(sum |F1|^2 sum |F2|^2) over rings
r = round(|(u, v)|), r = 0 .. N/2; FIRE = N / q, q the first 1/7 crossing (linear between rings,
r >= 2), NaN if FRC(1) < 1/7 or no crossing.  Only tests/ and bench.py's CPU baseline use it.
"""
from __future__ import annotations

import numpy as np

TAPER = 0.25


def padded_size(w, h):
    n = 32
    while n < max(w, h):
        n *= 2
    return n


def tukey(n):
    a = TAPER * (n - 1) * 0.5
    i = np.arange(n, dtype=np.float64)
    x = np.minimum(i, n - 1 - i)
    out = np.ones(n)
    if a > 0:
        m = x < a
        out[m] = 0.5 * (1 - np.cos(np.pi * x[m] / a))
    return out


def rings(N):
    f = np.fft.fftfreq(N, 1.0 / N).astype(np.int64)  # 0 .. N/2-1, -N/2 .. -1
    k = f[:, None] ** 2 + f[None, :] ** 2
    r = np.floor(np.sqrt(k)).astype(np.int64)
    r += (r + 1) ** 2 <= k
    r -= r * r > k
    return np.where(k > r * r + r, r + 1, r)


def curve(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    h, w = a.shape
    N = padded_size(w, h)
    win = tukey(h)[:, None] * tukey(w)[None, :]
    pa = np.zeros((N, N))
    pb = np.zeros((N, N))
    pa[:h, :w] = (a - a.mean()) * win
    pb[:h, :w] = (b - b.mean()) * win
    Fa, Fb = np.fft.fft2(pa), np.fft.fft2(pb)
    r = rings(N).ravel()
    R = N // 2 + 1
    keep = r < R
    c = np.bincount(r[keep], weights=np.real(Fa * np.conj(Fb)).ravel()[keep], minlength=R)
    s1 = np.bincount(r[keep], weights=(np.abs(Fa) ** 2).ravel()[keep], minlength=R)
    s2 = np.bincount(r[keep], weights=(np.abs(Fb) ** 2).ravel()[keep], minlength=R)
    with np.errstate(invalid="ignore", divide="ignore"):
        frc = np.where((s1 > 0) & (s2 > 0), c / np.sqrt(s1 * s2), 0.0)
    return frc, N


def fire(a, b, pixel_size=1.0):
    frc, N = curve(a, b)
    for r in range(1, len(frc)):
        if frc[r] < 1.0 / 7.0:
            if r < 2:
                return float("nan"), frc
            q = (r - 1) + (frc[r - 1] - 1.0 / 7.0) / (frc[r - 1] - frc[r])
            return N / q * pixel_size, frc
    return float("nan"), frc


def split_images(seed, h, w, cutoff, noise, n_spots=60):
    """Two images of one structure band-limited at `cutoff` cycles/pixel (a Gaussian spot field
    low-passed by an ideal disc filter) plus independent Gaussian noise of std `noise`."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    img = np.zeros((h, w))
    for _ in range(n_spots):
        px, py, amp = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(50, 200)
        img += amp * np.exp(-((xx - px) ** 2 + (yy - py) ** 2) / 2.0)
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.fftfreq(w)[None, :]
    img = np.real(np.fft.ifft2(np.fft.fft2(img) * (np.sqrt(fx ** 2 + fy ** 2) <= cutoff)))
    return img + rng.normal(0, noise, (h, w)), img + rng.normal(0, noise, (h, w))
