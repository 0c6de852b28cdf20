"""Seeded synthetic blinking-emitter stacks for the five benchmark workloads.

The reference ships no test data (its README points at external datasets), so every parity
test and every benchmark runs on stacks generated here.  The model:

* emitters: uniform in the field, or on random smooth filaments (cubic Bezier curves through
  random control points, emitters spaced uniformly in the curve parameter, Gaussian jitter of
  0.5 px, i.e. 50 nm at 100 nm pixels);
* PSF: pixel-integrated Gaussian, sigma 1.3 px (3-D: times a Gaussian in z, sigma 1 plane,
  normalised to 1 at the emitter's own depth);
* blinking: two-state Markov chain per emitter, off->on 0.05 and on->off 0.3 per frame, started
  from the stationary distribution;
* camera: 500 photons per on-emitter per frame, background 100, Poisson shot noise, Gaussian
  read noise sigma 2, offset 100, rounded and clipped to uint16.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

P_ON = 0.05
P_OFF = 0.3
PHOTONS = 500.0
BACKGROUND = 100.0
READ_NOISE = 2.0
OFFSET = 100.0
PSF_SIGMA = 1.3


@dataclass
class Workload:
    """One of the five benchmark workloads (shapes and eSRRF parameters)."""

    name: str
    width: int
    height: int
    frames: int
    magnification: int
    fwhm: float
    sensitivity: int
    planes: int = 1
    emitters: int = 0
    filaments: int = 0
    seed: int = 1234


WORKLOADS = {
    # 2-D FHT path, AVG, 64x64 x 100 frames, M5, radius 1.5, S1, 200 uniform emitters
    "fht64": Workload("fht64", 64, 64, 100, 5, 1.5, 1, emitters=200, filaments=0, seed=1235),
    # 2-D FHT path, AVG+VAR+TAC2, 512x512 x 500 frames in blocks of 100, M4, radius 1.5, S2
    "fht512": Workload("fht512", 512, 512, 500, 4, 1.5, 2, emitters=5000, filaments=40, seed=1236),
    # batched sweep input, 256x256 x 200 frames
    "sweep256": Workload("sweep256", 256, 256, 200, 4, 1.5, 1, emitters=5000, filaments=40,
                         seed=1237),
    # differentiable eSRRF, 256x256 x 100 frames, M4, AVG
    "adjoint256": Workload("adjoint256", 256, 256, 100, 4, 1.5, 1, emitters=5000, filaments=40,
                           seed=1238),
    # 3-D: 9 planes of 128x128 x 200 timepoints, M3, radius 1.5, S1, AVG+VAR
    "mfm3d": Workload("mfm3d", 128, 128, 200, 3, 1.5, 1, planes=9, emitters=2000, filaments=40,
                      seed=1239),
}


def _filament_points(rng, n_emitters, n_filaments, width, height, depth=None):
    """Emitter coordinates on random cubic Bezier filaments (+0.5 px Gaussian jitter)."""
    dims = 2 if depth is None else 3
    extent = np.array([width, height] + ([depth] if depth is not None else []), np.float64)
    per = np.full(n_filaments, n_emitters // n_filaments)
    per[: n_emitters - per.sum()] += 1
    pts = []
    for f in range(n_filaments):
        ctrl = rng.uniform(0.05, 0.95, size=(4, dims)) * extent
        t = rng.uniform(0.0, 1.0, size=(per[f], 1))
        b = ((1 - t) ** 3) * ctrl[0] + 3 * ((1 - t) ** 2) * t * ctrl[1] \
            + 3 * (1 - t) * (t ** 2) * ctrl[2] + (t ** 3) * ctrl[3]
        jitter = rng.normal(0.0, 0.5, size=b.shape)
        if dims == 3:
            jitter[:, 2] *= 0.2  # 0.5 px lateral jitter ~ 0.1 plane axially
        pts.append(b + jitter)
    return np.concatenate(pts, axis=0)


def _blinking(rng, n_emitters, n_frames):
    """Two-state Markov on/off states, [frames][emitters] bool."""
    on = rng.random(n_emitters) < P_ON / (P_ON + P_OFF)
    states = np.empty((n_frames, n_emitters), bool)
    for t in range(n_frames):
        states[t] = on
        u = rng.random(n_emitters)
        on = np.where(on, u >= P_OFF, u < P_ON)
    return states


def _pixel_integrated(centres, n, sigma, half=5):
    """Per-emitter 1-D pixel-integrated Gaussian profiles over a window of 2*half+1 pixels."""
    base = np.floor(centres).astype(np.int64) - half
    idx = base[:, None] + np.arange(2 * half + 1)[None, :]
    lo = (idx - centres[:, None]) / (sigma * math.sqrt(2.0))
    hi = (idx + 1 - centres[:, None]) / (sigma * math.sqrt(2.0))
    from scipy.special import erf

    prof = 0.5 * (erf(hi) - erf(lo))
    valid = (idx >= 0) & (idx < n)
    return np.clip(idx, 0, n - 1), prof * valid


def _camera(rng, expected):
    counts = rng.poisson(expected).astype(np.float64)
    counts += rng.normal(0.0, READ_NOISE, size=counts.shape) + OFFSET
    return np.clip(np.rint(counts), 0, 65535).astype(np.uint16)


def make_stack(workload: str | Workload, frames: int | None = None) -> np.ndarray:
    """Generate the uint16 stack of a workload: [frames][H][W] (2-D) or [frames][P][H][W]."""
    wl = WORKLOADS[workload] if isinstance(workload, str) else workload
    n_frames = wl.frames if frames is None else frames
    rng = np.random.default_rng(wl.seed)
    W, H = wl.width, wl.height
    if wl.planes > 1:
        return _make_stack_3d(rng, wl, n_frames)
    if wl.filaments:
        xy = _filament_points(rng, wl.emitters, wl.filaments, W, H)
    else:
        xy = rng.uniform(0, 1, size=(wl.emitters, 2)) * np.array([W, H])
    states = _blinking(rng, len(xy), n_frames)
    ix, px = _pixel_integrated(xy[:, 0], W, PSF_SIGMA)
    iy, py = _pixel_integrated(xy[:, 1], H, PSF_SIGMA)
    out = np.empty((n_frames, H, W), np.uint16)
    for t in range(n_frames):
        on = np.nonzero(states[t])[0]
        img = np.full(H * W, BACKGROUND)
        if len(on):
            vals = PHOTONS * py[on][:, :, None] * px[on][:, None, :]
            flat = iy[on][:, :, None] * W + ix[on][:, None, :]
            img += np.bincount(flat.ravel(), weights=vals.ravel(), minlength=H * W)
        out[t] = _camera(rng, img.reshape(H, W))
    return out


def _make_stack_3d(rng, wl, n_frames):
    W, H, P = wl.width, wl.height, wl.planes
    xyz = _filament_points(rng, wl.emitters, wl.filaments, W, H, depth=P)
    states = _blinking(rng, len(xyz), n_frames)
    ix, px = _pixel_integrated(xyz[:, 0], W, PSF_SIGMA)
    iy, py = _pixel_integrated(xyz[:, 1], H, PSF_SIGMA)
    zc = np.arange(P)[None, :] + 0.5
    pz = np.exp(-((zc - xyz[:, 2:3]) ** 2) / (2 * 1.0 ** 2))  # [emitters][planes]
    out = np.empty((n_frames, P, H, W), np.uint16)
    for t in range(n_frames):
        on = np.nonzero(states[t])[0]
        img = np.full((P, H * W), BACKGROUND)
        if len(on):
            lat = PHOTONS * py[on][:, :, None] * px[on][:, None, :]
            flat = (iy[on][:, :, None] * W + ix[on][:, None, :]).ravel()
            for z in range(P):
                img[z] += np.bincount(flat, weights=(lat * pz[on, z][:, None, None]).ravel(),
                                      minlength=H * W)
        out[t] = _camera(rng, img.reshape(P, H, W))
    return out


def small_stack(seed: int, frames: int, height: int, width: int, emitters: int = 12,
                planes: int = 1) -> np.ndarray:
    """A small blinking-emitter stack for parity tests (same model, any shape)."""
    wl = Workload("small", width, height, frames, 1, 1.5, 1, planes=planes, emitters=emitters,
                  filaments=0 if planes == 1 else 2, seed=seed)
    if planes > 1:
        return make_stack(wl)
    return make_stack(wl)
