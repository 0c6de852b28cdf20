"""TEST INFRASTRUCTURE ONLY -- float64 restatement of the SQUIRREL error map of
ErrorMapLiveSRRF.java (optimise, :81-150; calculateErrorMap, :153-193; calculateAlphaBeta,
:206-239), the checker for esrrf_squirrel.

The blur restates ImageJ's FloatProcessor.blurGaussian as the reference calls it (GaussianBlur,
accuracy 0.01: kernel radius ceil(sigma sqrt(-2 ln 0.01)) + 1, normalised sampled Gaussian, edge
pixels replicated; ImageJ's kernel-tail smoothing and large-sigma down-sampling are not restated,
and ImageJ is not in the reference tree, so parity with Fiji's own numbers is unpinned).  The sigma
search restates Brent's localmin (R. P. Brent, 1973) as commons-math3's BrentOptimizer runs it:
start at the interval's midpoint, stop when |x - m| <= 2 tol - (b - a) / 2, tol = 1e-10 |x| +
1e-14.  Only tests/ use this module.
"""
from __future__ import annotations

import math

import numpy as np


def kernel_radius(sigma):
    return 0 if not sigma > 0 else int(math.ceil(sigma * math.sqrt(-2.0 * math.log(0.01)))) + 1


def blur(img, sigma):
    img = np.asarray(img, np.float64)
    r = kernel_radius(sigma)
    if r == 0:
        return img.copy()
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * x * x / (sigma * sigma))
    k /= k.sum()
    pad = np.pad(img, ((0, 0), (r, r)), mode="edge")
    tmp = sum(k[i] * pad[:, i:i + img.shape[1]] for i in range(2 * r + 1))
    pad = np.pad(tmp, ((r, r), (0, 0)), mode="edge")
    return sum(k[i] * pad[i:i + img.shape[0], :] for i in range(2 * r + 1))


def fit(B, ref):
    """calculateAlphaBeta with blurred ones = 1, then RMSE and the Pearson coefficient of
    alpha B + beta against ref."""
    b, r = B.ravel(), np.asarray(ref, np.float64).ravel()
    n = b.size
    sb, sbb, sbr, sr, srr = b.sum(), (b * b).sum(), (b * r).sum(), r.sum(), (r * r).sum()
    den = n * sbb - sb * sb
    alpha = (n * sbr - sr * sb) / den if den != 0 else 0.0
    beta = sr / n - alpha * sb / n
    rmse = math.sqrt(np.mean((alpha * b + beta - r) ** 2))
    vr = n * srr - sr * sr
    ppmcc = (math.copysign(1.0, alpha) * (n * sbr - sb * sr) / math.sqrt(den * vr)) if den > 0 and vr > 0 else 0.0
    return alpha, beta, rmse, ppmcc


def brent(f, lo, hi, rel=1e-10, abs_tol=1e-14, max_evals=1000):
    c = 0.5 * (3.0 - math.sqrt(5.0))
    a, b = lo, hi
    x = w = v = 0.5 * (lo + hi)
    fx = fw = fv = f(x)
    best_x, best_f = x, fx
    d = e = 0.0
    evals = 1
    while evals < max_evals:
        m = 0.5 * (a + b)
        tol1 = rel * abs(x) + abs_tol
        tol2 = 2.0 * tol1
        if abs(x - m) <= tol2 - 0.5 * (b - a):
            break
        golden = True
        if abs(e) > tol1:
            r = (x - w) * (fx - fv)
            q = (x - v) * (fx - fw)
            p = (x - v) * q - (x - w) * r
            q = 2.0 * (q - r)
            if q > 0:
                p = -p
            else:
                q = -q
            r, e = e, d
            if abs(p) < abs(0.5 * q * r) and q * (a - x) < p < q * (b - x):
                d = p / q
                u = x + d
                if u - a < tol2 or b - u < tol2:
                    d = tol1 if x <= m else -tol1
                golden = False
        if golden:
            e = (b - x) if x < m else (a - x)
            d = c * e
        u = x + (d if abs(d) >= tol1 else (tol1 if d > 0 else -tol1))
        fu = f(u)
        evals += 1
        if fu < best_f:
            best_x, best_f = u, fu
        if fu <= fx:
            if u < x:
                b = x
            else:
                a = x
            v, fv, w, fw, x, fx = w, fw, x, fx, u, fu
        else:
            if u < x:
                a = u
            else:
                b = u
            if fu <= fw or w == x:
                v, fv, w, fw = w, fw, u, fu
            elif fu <= fv or v == x or v == w:
                v, fv = u, fu
    return best_x


def squirrel(sr, ref, M, fixed_sigma=None, crop=0):
    """One image: dict(sigma, alpha, beta, rse, rsp, error_map)."""
    sr = np.asarray(sr, np.float64)
    ref = np.asarray(ref, np.float64)
    if crop:
        c = crop * M
        sr, ref = sr[c:-c, c:-c], ref[c:-c, c:-c]
    smax = float(np.float32(np.float32(4.0) / np.float32(2.35482)) * np.float32(M))  # Java float
    if fixed_sigma is not None:
        sigma = float(np.float32(fixed_sigma) * np.float32(M))
    else:
        sigma = brent(lambda s: fit(blur(sr, s), ref)[2], 0.0, smax)
    B = blur(sr, sigma)
    alpha, beta, rmse, ppmcc = fit(B, ref)
    return dict(sigma=sigma, alpha=alpha, beta=beta, rse=rmse, rsp=ppmcc,
                error_map=np.abs(ref - (alpha * B + beta)))
