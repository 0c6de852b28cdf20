"""TEST INFRASTRUCTURE ONLY -- ctypes front end of the CPU checkers.

Two libraries, neither part of the product:

* ``oracle/liboracle.so``: our C restatement of the reference eSRRF path (esrrf_oracle.c),
  FP32 (reference expression order) and FP64 variants.
* ``oracle/_ref/libesrrf_ref.so``: the reference's own OpenCL C kernels
  (resources/liveSRRF_noInterpolation.cl, liveSRRF.cl, live3DSRRF.cl) compiled as C++ on the
  host and replayed in LiveSRRF_CL.java's launch order.  Built only where the reference tree is
  present; ``ref_available()`` says whether it is loadable here.

Only tests/, ``__graft_entry__.smoke()`` and the bench's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_RESTATEMENT = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libesrrf_ref.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_lib = None
_ref = None


def build(reference_root: str | None = None) -> None:
    """Compile the restatement, and the reference-kernel replay when the reference exists.

    The reference tree is ``reference_root`` or the ``ESRRF_REFERENCE_DIR`` environment
    variable; with neither, or without the tree there, only the restatement is built.
    """
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
    ref = reference_root or os.environ.get("ESRRF_REFERENCE_DIR", "")
    if ref and os.path.isfile(os.path.join(ref, "resources", "liveSRRF_noInterpolation.cl")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_f32p)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_RESTATEMENT):
            build()
        _lib = ctypes.CDLL(_RESTATEMENT)
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(_REF)
    return _ref


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


# ------------------------------------------------------------------ restatement (ours)


def fht_interpolate(raw, magnification: int, scale_mode: int = 0) -> np.ndarray:
    """Fourier interpolation of a stack [n][h][w] -> [n][h*M][w*M] (FourierInterpolation.java)."""
    raw = _f32(raw)
    n, h, w = raw.shape
    out = np.empty((n, h * magnification, w * magnification), np.float32)
    L = lib()
    L.orc_fht_interpolate.restype = ctypes.c_int
    _check(L.orc_fht_interpolate(_ptr(raw), n, w, h, magnification, scale_mode, _ptr(out)),
           "orc_fht_interpolate")
    return out


def robx(img):
    img = _f32(img)
    h, w = img.shape
    gx = np.empty_like(img)
    gy = np.empty_like(img)
    lib().orc_robx_f32(_ptr(img), w, h, _ptr(gx), _ptr(gy))
    return gx, gy


def fht_block(interp, magnification, fwhm, sensitivity, int_weighting=True, drift_x=None,
              drift_y=None, precision="f32") -> np.ndarray:
    """One SR block of the FHT path on interpolated frames [n][HM][WM] -> [4][HM][WM]."""
    interp = _f32(interp)
    n, HM, WM = interp.shape
    out = np.empty((4, HM, WM), np.float32)
    fn = getattr(lib(), f"orc_fht_block_{precision}")
    _check(fn(_ptr(interp), n, WM, HM, magnification, ctypes.c_float(fwhm), int(sensitivity),
              int(bool(int_weighting)), _ptr(_f32(drift_x)), _ptr(_f32(drift_y)), _ptr(out)),
           "orc_fht_block")
    return out


def bic_block(frames, magnification, fwhm, sensitivity, int_weighting=True, mp_correction=True,
              drift_x=None, drift_y=None, precision="f32") -> np.ndarray:
    """One SR block of the 2-D bicubic path on raw frames [n][H][W] -> [4][H*M][W*M]."""
    frames = _f32(frames)
    n, H, W = frames.shape
    out = np.empty((4, H * magnification, W * magnification), np.float32)
    fn = getattr(lib(), f"orc_bic_block_{precision}")
    _check(fn(_ptr(frames), n, W, H, magnification, ctypes.c_float(fwhm), int(sensitivity),
              int(bool(int_weighting)), int(bool(mp_correction)), _ptr(_f32(drift_x)),
              _ptr(_f32(drift_y)), _ptr(out)), "orc_bic_block")
    return out


def block3d(planes, magnification, fwhm, sensitivity, theta_deg, shift_x, shift_y,
            int_weighting=True, mp_correction=True, drift_x=None, drift_y=None,
            precision="f32") -> np.ndarray:
    """One SR block of the 3-D path on planes [n][P][h][w] -> [4][P*M][h*M][w*M]."""
    planes = _f32(planes)
    n, P, H, W = planes.shape
    M = magnification
    out = np.empty((4, P * M, H * M, W * M), np.float32)
    fn = getattr(lib(), f"orc_3d_block_{precision}")
    _check(fn(_ptr(planes), n, P, W, H, M, ctypes.c_float(fwhm), int(sensitivity),
              int(bool(int_weighting)), int(bool(mp_correction)), _ptr(_f32(theta_deg)),
              _ptr(_f32(shift_x)), _ptr(_f32(shift_y)), _ptr(_f32(drift_x)),
              _ptr(_f32(drift_y)), _ptr(out)), "orc_3d_block")
    return out


def mfm_reshape(frames, n_planes, roi, coeff, background) -> np.ndarray:
    frames = _f32(frames)
    n, H, W = frames.shape
    out = np.empty((n, n_planes, H // 3, W // 3), np.float32)
    _check(lib().orc_mfm_reshape(_ptr(frames), n, W, H, n_planes, _ptr(_f32(roi)),
                                 _ptr(_f32(coeff)), ctypes.c_float(background), _ptr(out)),
           "orc_mfm_reshape")
    return out


# ------------------------------------------------------------------ reference kernels


def ref_fht_block(interp, magnification, fwhm, sensitivity, int_weighting=True, drift_x=None,
                  drift_y=None, frames_per_load=0) -> np.ndarray:
    interp = _f32(interp)
    n, HM, WM = interp.shape
    out = np.empty((4, HM, WM), np.float32)
    _check(ref().ref_fht_block(_ptr(interp), n, WM, HM, magnification, ctypes.c_float(fwhm),
                               int(sensitivity), int(frames_per_load), int(bool(int_weighting)),
                               _ptr(_f32(drift_x)), _ptr(_f32(drift_y)), _ptr(out)),
           "ref_fht_block")
    return out


def ref_fht_gradient(frame):
    frame = _f32(frame)
    HM, WM = frame.shape
    gx = np.empty_like(frame)
    gy = np.empty_like(frame)
    _check(ref().ref_fht_gradient(_ptr(frame), WM, HM, _ptr(gx), _ptr(gy)), "ref_fht_gradient")
    return gx, gy


def ref_bic_block(frames, magnification, fwhm, sensitivity, int_weighting=True,
                  mp_correction=True, drift_x=None, drift_y=None, frames_per_load=0):
    frames = _f32(frames)
    n, H, W = frames.shape
    M = magnification
    out = np.empty((4, H * M, W * M), np.float32)
    mp = np.empty((3, M, M), np.float32)
    _check(ref().ref_bic_block(_ptr(frames), n, W, H, M, ctypes.c_float(fwhm), int(sensitivity),
                               int(frames_per_load), int(bool(int_weighting)),
                               int(bool(mp_correction)), _ptr(_f32(drift_x)),
                               _ptr(_f32(drift_y)), _ptr(out), _ptr(mp)), "ref_bic_block")
    return out


def ref_3d_block(planes, magnification, fwhm, sensitivity, theta_deg, shift_x, shift_y,
                 int_weighting=True, mp_correction=True, dim_ratio=2.5, drift_x=None,
                 drift_y=None, frames_per_load=0):
    planes = _f32(planes)
    n, P, H, W = planes.shape
    M = magnification
    out = np.empty((4, P * M, H * M, W * M), np.float32)
    _check(ref().ref_3d_block(_ptr(planes), n, P, W, H, M, ctypes.c_float(fwhm),
                              int(sensitivity), int(frames_per_load), int(bool(int_weighting)),
                              int(bool(mp_correction)), _ptr(_f32(theta_deg)),
                              _ptr(_f32(shift_x)), _ptr(_f32(shift_y)), ctypes.c_float(dim_ratio),
                              _ptr(_f32(drift_x)), _ptr(_f32(drift_y)), _ptr(out)),
           "ref_3d_block")
    return out


# ------------------------------------------------------------------ FFT form of the interpolation


def _mirror_src(c, n, out_dim):
    scale = int(np.ceil(out_dim / n))
    if scale % 2 == 0:
        scale += 1
    roi = (scale * n - out_dim) // 2
    pos = c + roi
    tile = pos // n
    i = pos - tile * n
    rel = tile - (scale - 1) // 2
    return i if rel % 2 == 0 else n - 1 - i


def fht_interpolate_fft(raw, magnification: int, scale_mode: int = 0) -> np.ndarray:
    """Same map as ``fht_interpolate`` (FourierInterpolation.java:12-73) evaluated with numpy's
    FFT: DHT = Re(F) - Im(F) of the 2-D DFT, spectral remap, inverse DHT on the magnified canvas.
    Used where the definition-based form is too slow (the bench's CPU baseline)."""
    raw = np.asarray(raw, np.float64)
    n, h, w = raw.shape
    M = magnification
    N = max(1 << int(np.ceil(np.log2(w))), 1 << int(np.ceil(np.log2(h))))
    NM = N * M
    WM, HM = w * M, h * M
    xroi, yroi = (NM - WM) // 2, (NM - HM) // 2
    sx = np.array([_mirror_src(c, w, N) for c in range(N)])
    sy = np.array([_mirror_src(c, h, N) for c in range(N)])
    kmap = np.array([p if p < N // 2 else p + (M - 1) * N for p in range(N)])
    s = 1.0 / (N * N) if scale_mode == 0 else 1.0 / (NM * NM)
    out = np.empty((n, HM, WM), np.float32)
    for f in range(n):
        X = raw[f][sy][:, sx]
        F = np.fft.fft2(X)
        Hs = F.real - F.imag
        big = np.zeros((NM, NM))
        big[np.ix_(kmap, kmap)] = Hs
        G = np.fft.fft2(big)
        out[f] = ((G.real - G.imag) * s)[yroi:yroi + HM, xroi:xroi + WM]
    return out
