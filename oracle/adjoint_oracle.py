"""TEST INFRASTRUCTURE ONLY -- FP64 reference for the differentiable eSRRF loss.

The fidelity loss (no counterpart in the reference code; it follows the SQUIRREL-style error of
ErrorMapLiveSRRF.java:81-233 -- Gaussian re-blur of the reconstruction, linear intensity fit
against the wide-field image):

    R      = AVG reconstruction of the 2-D FHT path (intensity weighting on, zero drift),
             R(q) = (1/T) sum_t I_t(q) C_t(q)^S,  S real,  C_t = CGLH / sum of weights
    B      = G_sigma * R           (sampled Gaussian, normalised, radius ceil(4 sigma), zero padding)
    D      = M x M box average of B -> input grid
    F      = (1/T) sum_t raw_t      (frame average of the input)
    alpha, beta = least-squares fit of F ~ alpha D + beta
    loss   = mean((alpha D + beta - F)^2)

Everything here is float64 (interpolation by numpy FFT, Roberts cross, RGC per tap), so central
finite differences of `loss()` give the FP64 reference gradient the GPU adjoint is checked
against.  Only tests/ and the bench's checker legs use this module.
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def interpolate_f64(raw, M):
    """FourierInterpolation.java's map in float64 (same as oracle.fht_interpolate_fft)."""
    raw = np.asarray(raw, np.float64)
    n, h, w = raw.shape
    N = max(1 << int(np.ceil(np.log2(w))), 1 << int(np.ceil(np.log2(h))))
    NM = N * M
    WM, HM = w * M, h * M
    xroi, yroi = (NM - WM) // 2, (NM - HM) // 2
    sx = np.array([O._mirror_src(c, w, N) for c in range(N)])
    sy = np.array([O._mirror_src(c, h, N) for c in range(N)])
    kmap = np.array([p if p < N // 2 else p + (M - 1) * N for p in range(N)])
    out = np.empty((n, HM, WM))
    for f in range(n):
        X = raw[f][sy][:, sx]
        F = np.fft.fft2(X)
        big = np.zeros((NM, NM))
        big[np.ix_(kmap, kmap)] = F.real - F.imag
        G = np.fft.fft2(big)
        out[f] = ((G.real - G.imag) / (N * N))[yroi:yroi + HM, xroi:xroi + WM]
    return out


def geometry(M, fwhm):
    """Tap offsets and weights of the FHT path (LiveSRRF_CL.java:491-500; float constants)."""
    sigma = np.float32(fwhm) / np.float32(2.354)
    Mf = np.float32(M)
    tSS = float(np.float32(np.float32(np.float32(np.float32(2) * sigma) * Mf) * sigma) * Mf)
    tSO = float((np.float32(2) * sigma + np.float32(1)) * Mf)
    R = Mf * (np.float32(int(np.float32(2) * sigma)) + np.float32(1))
    r0, r1 = -int(R), int(R + 1)
    taps = []
    for j in range(r0, r1 + 1):
        for i in range(r0, r1 + 1):
            d = np.sqrt(np.float32(i * i + j * j))
            if d != 0 and d <= np.float32(tSO):
                taps.append((i, j, float(np.sqrt(i * i + j * j))))
    return taps, tSS


def cglh_f64(I, M, fwhm):
    """C_t = CGLH / sum of weights per frame, float64 (liveSRRF_noInterpolation.cl:245-349)."""
    T, H, W = I.shape
    taps, tSS = geometry(M, fwhm)
    out = np.empty_like(I)
    for t in range(T):
        p = I[t]
        x0 = np.r_[0, np.arange(W - 1)]
        y0 = np.r_[0, np.arange(H - 1)]
        gx = p[y0, :] - p[:, x0] + p - p[y0][:, x0]
        gy = -p[y0, :] + p[:, x0] + p - p[y0][:, x0]
        num = np.zeros((H, W))
        den = np.zeros((H, W))
        yy, xx = np.mgrid[0:H, 0:W]
        for (i, j, d) in taps:
            X, Y = xx + i, yy + j
            ok = (X >= 0) & (X < W) & (Y >= 0) & (Y < H)
            Xc, Yc = np.clip(X, 0, W - 1), np.clip(Y, 0, H - 1)
            Gx = gx[Yc, np.minimum(Xc + 1, W - 1)]
            Gy = gy[np.minimum(Yc + 1, H - 1), Xc]
            w = (d * np.exp(-(d * d) / tSS)) ** 4
            den += np.where(ok, w, 0.0)
            dot = Gx * i + Gy * j
            gm = np.sqrt(Gx * Gx + Gy * Gy)
            with np.errstate(invalid="ignore", divide="ignore"):
                dk = np.abs(Gy * i - Gx * j) / gm
            dk = np.where(np.isnan(dk), d, dk)
            num += np.where(ok & (dot < 0), (1 - dk / d) * w, 0.0)
        with np.errstate(invalid="ignore", divide="ignore"):
            out[t] = num / den
    return out


def gauss1d(sigma):
    r = int(np.ceil(4 * sigma))
    u = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-u * u / (2 * sigma * sigma))
    return k / k.sum()


def blur(img, sigma):
    k = gauss1d(sigma)
    r = len(k) // 2
    pad = np.pad(img, ((0, 0), (r, r)))
    tmp = sum(k[i] * pad[:, i:i + img.shape[1]] for i in range(len(k)))
    pad = np.pad(tmp, ((r, r), (0, 0)))
    return sum(k[i] * pad[i:i + img.shape[0], :] for i in range(len(k)))


def loss(raw, M, fwhm, S, sigma_b, return_parts=False):
    raw = np.asarray(raw, np.float64)
    T, h, w = raw.shape
    I = interpolate_f64(raw, M)
    C = cglh_f64(I, M, fwhm)
    with np.errstate(invalid="ignore", divide="ignore"):
        Cs = np.where(C > 0, np.power(np.where(C > 0, C, 1.0), S), 0.0)
    R = (I * Cs).mean(axis=0)
    B = blur(R, sigma_b)
    D = B.reshape(h, M, w, M).mean(axis=(1, 3))
    F = raw.mean(axis=0)
    d, f = D.ravel(), F.ravel()
    dm, fm = d.mean(), f.mean()
    alpha = ((d - dm) * (f - fm)).sum() / ((d - dm) ** 2).sum()
    beta = fm - alpha * dm
    L = float(np.mean((alpha * D + beta - F) ** 2))
    if return_parts:
        return L, dict(R=R, D=D, F=F, alpha=alpha, beta=beta, C=C, I=I)
    return L


def fd_gradient(raw, M, fwhm, S, sigma_b, pixels=(), h=1e-3):
    """Central differences (step h) of the FP64 loss w.r.t. radius, sensitivity, blur sigma and
    the listed input pixels (t, y, x)."""
    raw = np.asarray(raw, np.float64)
    g = {}
    g["fwhm"] = (loss(raw, M, fwhm + h, S, sigma_b) - loss(raw, M, fwhm - h, S, sigma_b)) / (2 * h)
    g["S"] = (loss(raw, M, fwhm, S + h, sigma_b) - loss(raw, M, fwhm, S - h, sigma_b)) / (2 * h)
    g["sigma"] = (loss(raw, M, fwhm, S, sigma_b + h) - loss(raw, M, fwhm, S, sigma_b - h)) / (2 * h)
    px = {}
    for (t, y, x) in pixels:
        a = raw.copy()
        a[t, y, x] += h
        lp = loss(a, M, fwhm, S, sigma_b)
        a[t, y, x] -= 2 * h
        lm = loss(a, M, fwhm, S, sigma_b)
        px[(t, y, x)] = (lp - lm) / (2 * h)
    g["pixels"] = px
    return g
