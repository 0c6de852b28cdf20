"""Generates the golden fixtures in this folder from the reference's own kernels.

The reference ships no test vectors, so these are made by running the reference's OpenCL C
kernel sources (resources/liveSRRF_noInterpolation.cl, liveSRRF.cl, live3DSRRF.cl), compiled on
the host by oracle/Makefile (`make -C oracle ref`), in LiveSRRF_CL.java's launch order, on small
seeded blinking-emitter stacks.  FHT-path inputs are Fourier-interpolated by our restatement
(the reference's transform, nanoj.core2.NanoJFHT, is not vendored), and stored with the case so
the fixture pins the kernels independently of that stage.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "nanoj-esrrf_b200"))

from esrrf import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name, kind, (frames, h, w), magnification, fwhm, sensitivity, int_weighting, mp, drift, seed
CASES = [
    ("fht_m3_s2", "fht", (8, 20, 24), 3, 1.5, 2, True, False, False, 11),
    ("fht_m5_s1_noint", "fht", (6, 16, 16), 5, 1.5, 1, False, False, False, 12),
    ("fht_m2_r3_s3", "fht", (7, 24, 20), 2, 3.0, 3, True, False, False, 13),
    ("fht_m4_drift", "fht", (6, 16, 16), 4, 1.5, 1, True, False, True, 14),
    ("bic_m4_mp", "bic", (8, 20, 20), 4, 1.5, 1, True, True, False, 15),
    ("bic_m3_drift_nomp", "bic", (6, 18, 22), 3, 2.0, 2, True, False, True, 16),
    ("3d_m3_mp", "3d", (5, 12, 12), 3, 1.5, 1, True, True, False, 17),
]


def make_case(name, kind, shape, M, fwhm, sens, intw, mp, drift, seed):
    rng = np.random.default_rng(seed)
    n, h, w = shape
    dx = dy = None
    if drift:
        dx = (0.3 * rng.standard_normal(n)).astype(np.float32)
        dy = (0.3 * rng.standard_normal(n)).astype(np.float32)
    rec = dict(kind=kind, magnification=M, fwhm=np.float32(fwhm), sensitivity=sens,
               int_weighting=int(intw), mp_correction=int(mp))
    if dx is not None:
        rec.update(drift_x=dx, drift_y=dy)
    if kind == "fht":
        raw = synth.small_stack(seed, n, h, w).astype(np.float32)
        interp = O.fht_interpolate(raw, M)
        out = O.ref_fht_block(interp, M, fwhm, sens, int_weighting=intw, drift_x=dx, drift_y=dy,
                              frames_per_load=3)
        rec.update(raw=raw, interp=interp, out=out)
    elif kind == "bic":
        raw = synth.small_stack(seed, n, h, w).astype(np.float32)
        out = O.ref_bic_block(raw, M, fwhm, sens, int_weighting=intw, mp_correction=mp,
                              drift_x=dx, drift_y=dy, frames_per_load=3)
        rec.update(raw=raw, out=out)
    else:
        P = 4
        planes = synth.small_stack(seed, n, h, w, planes=P).astype(np.float32)
        theta = np.array([0.4, -0.8, 0.0, 1.1], np.float32)
        sx = np.array([0.1, -0.2, 0.0, 0.3], np.float32)
        sy = np.array([-0.1, 0.25, 0.0, 0.15], np.float32)
        out = O.ref_3d_block(planes, M, fwhm, sens, theta, sx, sy, int_weighting=intw,
                             mp_correction=mp, frames_per_load=2)
        rec.update(raw=planes, theta=theta, shift_x=sx, shift_y=sy, out=out)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **rec)
    return rec


def main():
    if not O.ref_available():
        O.build()
    if not O.ref_available():
        raise SystemExit("reference kernels not built: set ESRRF_REFERENCE_DIR to the reference tree")
    for c in CASES:
        make_case(*c)
        print("wrote", c[0])


if __name__ == "__main__":
    main()
