"""Python front end of libesrrf, the B200 eSRRF engine.

``LiveSRRF_CL`` mirrors the reference's device-engine class nanoj.liveSRRF.LiveSRRF_CL
(src/nanoj/liveSRRF/LiveSRRF_CL.java) member for member, over the C ABI in include/esrrf.h, so
that code written against the Fiji plugin's engine reads the same here.  ``esrrf_stack`` is a
one-call functional form used by the benchmark and the parity tests.

There is no CPU fallback: importing this package on a machine without the built library raises,
and every call that reaches the GPU raises ``EsrrfError`` on failure.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import EsrrfError, EsrrfParams, lib

__all__ = ["LiveSRRF_CL", "EsrrfError", "EsrrfParams", "esrrf_stack", "lib", "default_params"]

# Keys of the 3-D calibration table that LiveSRRF_CL.initialise reads (LiveSRRF_CL.java:212-220).
CALIB_KEYS = ("X-shift (pixels)", "Y-shift (pixels)", "Theta (degrees)", "Axial positions",
              "ROI #", "Intensity scaling", "Background level (ADC)")


def default_params() -> EsrrfParams:
    p = EsrrfParams()
    lib().esrrf_default_params(ctypes.byref(p))
    return p


class LiveSRRF_CL:
    """Mirror of nanoj.liveSRRF.LiveSRRF_CL over libesrrf (one CUDA stream per instance)."""

    nReconstructions = 3  # AVG, VAR, TAC2 (LiveSRRF_CL.java:51)
    gradientMag = 2       # 2x gradient grid of the bicubic paths (LiveSRRF_CL.java:45)

    def __init__(self, DEBUG: bool = False):
        self.DEBUG = DEBUG
        self._h = ctypes.c_void_p()
        self._keep = []
        self.allCLdevices: list[str] = []
        self.imsSRRF: np.ndarray | None = None
        self.widthS = self.heightS = 0
        self.nPlanes = self.nPlanesM = 1
        self._shape = None
        self._frame_shape = None

    # -- LiveSRRF_CL.checkDevices (LiveSRRF_CL.java:111-155)
    def checkDevices(self) -> list[str]:
        n = ctypes.c_int(0)
        lib().esrrf_device_count(ctypes.byref(n))
        names = []
        for d in range(n.value):
            buf = ctypes.create_string_buffer(256)
            sms, clk = ctypes.c_int(), ctypes.c_int()
            _lib.check(None, lib().esrrf_device_info(d, buf, 256, ctypes.byref(sms),
                                                     ctypes.byref(clk)))
            names.append(buf.value.decode())
        self.allCLdevices = names
        return names

    # -- LiveSRRF_CL.initialise (LiveSRRF_CL.java:159-264)
    def initialise(self, width, height, magnification, fwhm, sensitivity, nFramesOnGPU,
                   nFrameForSRRF, blockLength=20000, chosenDevice=None, intWeighting=True,
                   doMPmapCorrection=False, doFHTinterpolation=True, calibTable3DSRRF=None,
                   axialOffset=0.0, pixelSize=0.1, kernel="fused", framesPerLaunch=0,
                   fhtScale="mean_preserving"):
        """Same arguments as the reference.  ``calibTable3DSRRF``: the calibration table as a path
        (read by calibration.load_calibration_table: ImageJ's text export of the table) or a
        mapping with the table's keys (CALIB_KEYS); ``None`` means 2-D.  As the reference does
        (LiveSRRF_CL.java:232-238), a table whose axial positions do not sum to zero replaces
        axialOffset by their regression slope; axialOffset and dimensionRatioXYvsZ are kept on the
        object."""
        from . import calibration as _cal

        self.release()
        if calibTable3DSRRF is not None and isinstance(calibTable3DSRRF, (str, bytes, os.PathLike)):
            calibTable3DSRRF = _cal.load_calibration_table(calibTable3DSRRF)
        if calibTable3DSRRF is not None:
            geo = _cal.table_geometry(calibTable3DSRRF, width, height, magnification, axialOffset,
                                      pixelSize)
            axialOffset = geo["axialOffset"]
            self.dimensionRatioXYvsZ = geo["dimensionRatioXYvsZ"]
        else:
            self.dimensionRatioXYvsZ = None
        self.axialOffset = float(axialOffset)
        p = default_params()
        p.width, p.height = int(width), int(height)
        p.magnification = int(magnification)
        p.fwhm = float(fwhm)
        p.sensitivity = int(sensitivity)
        p.n_frames_on_gpu = int(nFramesOnGPU)
        p.n_frame_for_srrf = int(nFrameForSRRF)
        p.block_length = int(blockLength)
        p.device = -1 if chosenDevice is None else int(chosenDevice)
        p.int_weighting = int(bool(intWeighting))
        p.mp_correction = int(bool(doMPmapCorrection))
        p.interp = 0 if doFHTinterpolation else 1
        p.fht_scale = {"mean_preserving": 0, "unitary_big": 1}[fhtScale]
        p.kernel = {"fused": 0, "plain": 1}[kernel]
        # "auto": measured by the library's autotuner (cached per parameter set)
        p.frames_per_launch = -1 if framesPerLaunch == "auto" else int(framesPerLaunch)
        p.axial_offset_nm = float(axialOffset)
        p.pixel_size_um = float(pixelSize)
        self._keep = []
        if calibTable3DSRRF is not None:
            t = calibTable3DSRRF
            arrs = {k: np.ascontiguousarray(np.asarray(t[k], np.float32)) for k in CALIB_KEYS
                    if k in t}
            n_planes = len(arrs["X-shift (pixels)"])
            p.n_planes = n_planes
            fptr = ctypes.POINTER(ctypes.c_float)
            p.roi = arrs["ROI #"].ctypes.data_as(fptr)
            p.theta_deg = arrs["Theta (degrees)"].ctypes.data_as(fptr)
            p.shift_x = arrs["X-shift (pixels)"].ctypes.data_as(fptr)
            p.shift_y = arrs["Y-shift (pixels)"].ctypes.data_as(fptr)
            p.intensity_coeff = arrs["Intensity scaling"].ctypes.data_as(fptr)
            p.background = float(arrs["Background level (ADC)"][0])
            self._keep = list(arrs.values())
        h = ctypes.c_void_p()
        _lib.check(None, lib().esrrf_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self._params = p
        wm, hm, pm = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(h, lib().esrrf_output_shape(h, ctypes.byref(wm), ctypes.byref(hm),
                                               ctypes.byref(pm)))
        self._shape = (wm.value, hm.value, pm.value)
        self._frame_shape = (int(height), int(width))
        M = int(magnification)
        self.widthS, self.heightS = wm.value // M, hm.value // M
        self.nPlanesM = pm.value
        self.nPlanes = max(1, pm.value // M) if calibTable3DSRRF is not None else 1

    # -- LiveSRRF_CL.loadDriftXYGPUbuffer (LiveSRRF_CL.java:583-595)
    def loadDriftXYGPUbuffer(self, driftX, driftY):
        dx = np.ascontiguousarray(driftX, np.float32)
        dy = np.ascontiguousarray(driftY, np.float32)
        fptr = ctypes.POINTER(ctypes.c_float)
        _lib.check(self._h, lib().esrrf_set_drift(self._h, dx.ctypes.data_as(fptr),
                                                  dy.ctypes.data_as(fptr), len(dx)))

    # -- LiveSRRF_CL.resetFramePosition (LiveSRRF_CL.java:955-960)
    def resetFramePosition(self):
        _lib.check(self._h, lib().esrrf_reset_frame_position(self._h))

    # -- LiveSRRF_CL.calculateSRRF (LiveSRRF_CL.java:636-746); True if cancelled
    def calculateSRRF(self, imsRawData) -> bool:
        a = np.asarray(imsRawData)
        if self._frame_shape is None:
            raise EsrrfError("calculateSRRF before initialise")
        if a.ndim == 2:  # one frame
            a = a[None]
        if a.ndim != 3 or tuple(a.shape[1:]) != self._frame_shape:
            raise EsrrfError(f"frames must be [n][{self._frame_shape[0]}][{self._frame_shape[1]}] "
                             f"(height, width of initialise), got {list(a.shape)}")
        if a.dtype == np.uint16:
            a = np.ascontiguousarray(a)
            rc = lib().esrrf_calculate_srrf_u16(self._h, a.ctypes.data_as(ctypes.c_void_p),
                                                a.shape[0])
        else:
            a = np.ascontiguousarray(a, np.float32)
            rc = lib().esrrf_calculate_srrf_f32(self._h, a.ctypes.data_as(ctypes.c_void_p),
                                                a.shape[0])
        if rc == 1:
            return True
        _lib.check(self._h, rc)
        return False

    # -- LiveSRRF_CL.readSRRFbuffer (LiveSRRF_CL.java:749-794)
    def readSRRFbuffer(self):
        wm, hm, pm = self._shape
        out = np.empty((4 * pm, hm, wm), np.float32)
        _lib.check(self._h, lib().esrrf_read_srrf(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        self.imsSRRF = out
        return out

    def readSRRFbufferAsync(self, out):
        """Queued read-back of the block into `out` (a C-contiguous float32 array of
        [4 x planesM][heightM][widthM], pinned for overlap), valid once finishQueue() returns;
        the next block can be pushed meanwhile (esrrf_read_srrf_async)."""
        if not (isinstance(out, np.ndarray) and out.dtype == np.float32 and out.flags.c_contiguous):
            raise EsrrfError("readSRRFbufferAsync needs a C-contiguous float32 array")
        wm, hm, pm = self._shape
        if out.size != 4 * pm * hm * wm:
            raise EsrrfError(f"output holds {out.size} floats, the block {4 * pm * hm * wm}")
        _lib.check(self._h, lib().esrrf_read_srrf_async(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        self._async_out = out

    # -- LiveSRRF_CL.readGradientBuffers (LiveSRRF_CL.java:797-879)
    def readGradientBuffers(self):
        wm, hm, pm = self._shape
        out = np.empty((2, hm, wm), np.float32)
        _lib.check(self._h, lib().esrrf_read_gradients(self._h, out.ctypes.data_as(ctypes.c_void_p),
                                                       ctypes.c_size_t(out.size)))
        return out

    # -- LiveSRRF_CL.readAlignedPixels (LiveSRRF_CL.java:881-906); 3-D only
    def readAlignedPixels(self):
        out = np.empty((self.nPlanes, self.heightS, self.widthS), np.float32)
        _lib.check(self._h, lib().esrrf_read_aligned_pixels(self._h, out.ctypes.data_as(ctypes.c_void_p),
                                                            ctypes.c_size_t(out.size)))
        return out

    # -- LiveSRRF_CL.readMPmaps (LiveSRRF_CL.java:909-935); bicubic and 3-D paths with MP correction
    def readMPmaps(self):
        M = int(self._params.magnification)
        n = 3 * (M if self._params.n_planes > 0 else 1)
        out = np.empty((n, M, M), np.float32)
        _lib.check(self._h, lib().esrrf_read_mp_maps(self._h, out.ctypes.data_as(ctypes.c_void_p),
                                                     ctypes.c_size_t(out.size)))
        return out

    # -- LiveSRRF_CL.finishQueue (LiveSRRF_CL.java:1009-1015)
    def finishQueue(self):
        _lib.check(self._h, lib().esrrf_finish_queue(self._h))

    def requestCancel(self):
        """Thread-safe counterpart of the reference's Escape-key polling."""
        _lib.check(self._h, lib().esrrf_request_cancel(self._h))

    def framesPerLaunch(self) -> int:
        """Frames one RGC launch processes (no reference counterpart: the reference launches per
        frame); 0 at initialise picks the default split."""
        f = ctypes.c_int()
        _lib.check(self._h, lib().esrrf_frames_per_launch(self._h, ctypes.byref(f)))
        return f.value

    def tuneReport(self) -> dict:
        """What the autotuner chose for this engine (esrrf_tune_report): source "measured",
        "cache" or "off", frames_per_launch, form and the candidates' times."""
        import json

        buf = ctypes.create_string_buffer(8192)
        _lib.check(self._h, lib().esrrf_tune_report(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def lastTiming(self):
        i, r, n = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
        _lib.check(self._h, lib().esrrf_last_timing(self._h, ctypes.byref(i), ctypes.byref(r),
                                                    ctypes.byref(n)))
        return i.value, r.value, n.value

    def setStream(self, stream_ptr):
        """Run on a caller-owned cudaStream_t (an int pointer value); None restores a private one."""
        _lib.check(self._h, lib().esrrf_set_stream(self._h, ctypes.c_void_p(stream_ptr or None)))

    def setTiming(self, on: bool):
        _lib.check(self._h, lib().esrrf_set_timing(self._h, int(bool(on))))

    @property
    def handle(self):
        return self._h

    # -- LiveSRRF_CL.release (LiveSRRF_CL.java:939-951)
    def release(self):
        if self._h:
            lib().esrrf_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def esrrf_stack(stack, magnification, fwhm, sensitivity, frames_per_block=None, gap=None,
                int_weighting=True, mp_correction=False, fht=True, drift=None, kernel="fused",
                frames_per_launch=0, calib3d=None, n_frames_on_gpu=None):
    """Rolling eSRRF over a stack, the loop of LiveSRRF_optimised_.run
    (gui/LiveSRRF_optimised_.java:276-389): blocks of ``frames_per_block`` frames starting every
    ``gap`` frames; returns [blocks][4*planesM][HM][WM] (AVG, VAR, TAC2, INT)."""
    a = np.asarray(stack)
    n = a.shape[0]
    nf = n if frames_per_block is None else min(n, int(frames_per_block))
    gap = nf if gap is None else int(gap)
    n_blocks = int((n - nf) / gap) + 1
    h, w = a.shape[-2], a.shape[-1]
    eng = LiveSRRF_CL()
    eng.initialise(w, h, magnification, fwhm, sensitivity, n_frames_on_gpu or nf, nf,
                   intWeighting=int_weighting, doMPmapCorrection=mp_correction,
                   doFHTinterpolation=fht, calibTable3DSRRF=calib3d, kernel=kernel,
                   framesPerLaunch=frames_per_launch)
    outs = []
    try:
        for r in range(n_blocks):
            eng.resetFramePosition()
            if drift is not None:
                eng.loadDriftXYGPUbuffer(drift[0][r * gap:r * gap + nf], drift[1][r * gap:r * gap + nf])
            if eng.calculateSRRF(a[r * gap:r * gap + nf]):
                raise EsrrfError("cancelled")
            outs.append(eng.readSRRFbuffer().copy())
    finally:
        eng.release()
    return np.stack(outs)


class Sweep:
    """Batched parameter sweep / rolling analysis (esrrf_sweep_*): every (magnification, radius,
    sensitivity, block) reconstruction of a stack in one captured CUDA graph per device.  Replaces
    the per-combination engine loop of ParametersSweep_.run (gui/ParametersSweep_.java:328-519) and
    the block loop of LiveSRRF_optimised_.run (gui/LiveSRRF_optimised_.java:276-389).
    ``interpolation``: "fht" or "bicubic" (the sweep's "Use FHT interpolation" option; the
    bicubic sweep applies the MP correction, as the reference's sweep does).
    ``drift``: (shift_x, shift_y), one shift per frame of the stack in raw pixels (the sweep's
    vibration correction, gui/ParametersSweep_.java:282-290), FHT sweep only.
    ``devices``: a list of CUDA ordinals to split the sweep across (``plan`` shows the split)."""

    def __init__(self, width, height, n_frames, magnifications, radii, sensitivities, blocks,
                 int_weighting=True, device=-1, interpolation="fht", drift=None, devices=None):
        self._h = None
        self._p = self._params(width, height, n_frames, magnifications, radii, sensitivities, blocks,
                               int_weighting, device, interpolation, drift, devices)
        h = ctypes.c_void_p()
        _lib.check(None, lib().esrrf_sweep_create(ctypes.byref(self._p), ctypes.byref(h)), sweep=True)
        self._h = h
        total = ctypes.c_size_t()
        offs = (ctypes.c_size_t * (len(self.mags) * len(self.radii)))()
        _lib.check(h, lib().esrrf_sweep_output_layout(h, ctypes.byref(total), offs), sweep=True)
        self.total = total.value
        self.offsets = list(offs)

    def _params(self, width, height, n_frames, magnifications, radii, sensitivities, blocks,
                int_weighting, device, interpolation, drift, devices):
        from ._lib import EsrrfSweepParams

        self.width, self.height, self.n_frames = int(width), int(height), int(n_frames)
        self.mags = np.ascontiguousarray(magnifications, np.int32)
        self.radii = np.ascontiguousarray(radii, np.float32)
        self.sens = np.ascontiguousarray(sensitivities, np.int32)
        blocks = np.asarray(blocks, np.int64).reshape(-1, 2)
        self.bstart = np.ascontiguousarray(blocks[:, 0], np.int32)
        self.blen = np.ascontiguousarray(blocks[:, 1], np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        fp = ctypes.POINTER(ctypes.c_float)
        self._drift = None
        if drift is not None:
            dx = np.ascontiguousarray(drift[0], np.float32).reshape(-1)
            dy = np.ascontiguousarray(drift[1], np.float32).reshape(-1)
            if dx.size != self.n_frames or dy.size != self.n_frames:
                raise EsrrfError("drift arrays must hold one shift per frame of the stack")
            self._drift = (dx, dy)
        self._devices = None if devices is None else np.ascontiguousarray(devices, np.int32)
        return EsrrfSweepParams(self.width, self.height, self.n_frames, len(self.mags),
                                self.mags.ctypes.data_as(ip), len(self.radii), self.radii.ctypes.data_as(fp),
                                len(self.sens), self.sens.ctypes.data_as(ip), len(self.bstart),
                                self.bstart.ctypes.data_as(ip), self.blen.ctypes.data_as(ip),
                                int(bool(int_weighting)), int(device),
                                {"fht": 0, "bicubic": 1}[interpolation],
                                self._drift[0].ctypes.data_as(fp) if self._drift else None,
                                self._drift[1].ctypes.data_as(fp) if self._drift else None,
                                0 if self._devices is None else len(self._devices),
                                self._devices.ctypes.data_as(ip) if self._devices is not None else None)

    @staticmethod
    def plan(width, height, n_frames, magnifications, radii, sensitivities, blocks, devices,
             interpolation="fht"):
        """The split esrrf_sweep_create would make across ``devices`` (host arithmetic only):
        (pair_device [n_mag * n_radius], block_device [n_blocks], device_cost [n_devices]);
        -1 = every device of the split, -2 = none."""
        self = Sweep.__new__(Sweep)
        p = self._params(width, height, n_frames, magnifications, radii, sensitivities, blocks, True, -1,
                         interpolation, None, devices)
        nP, nB = len(self.mags) * len(self.radii), len(self.bstart)
        pd = (ctypes.c_int * nP)()
        bd = (ctypes.c_int * nB)()
        dc = (ctypes.c_double * max(1, len(devices)))()
        _lib.check(None, lib().esrrf_sweep_plan(ctypes.byref(p), pd, bd, dc), sweep=True)
        return list(pd), list(bd), list(dc)[:len(devices)]

    def shard_count(self) -> int:
        n = ctypes.c_int()
        _lib.check(self._h, lib().esrrf_sweep_shard_count(self._h, ctypes.byref(n)), sweep=True)
        return n.value

    @property
    def handle(self):
        return self._h

    def launch_count(self) -> int:
        n = ctypes.c_int()
        _lib.check(self._h, lib().esrrf_sweep_launch_count(self._h, ctypes.byref(n)), sweep=True)
        return n.value

    def unpack(self, flat):
        """{(M, radius, S, (start, length)): [4][HM][WM]} views of a flat output buffer."""
        out = {}
        nS, nB = len(self.sens), len(self.bstart)
        for mi, M in enumerate(self.mags):
            P = self.height * M * self.width * M
            for ri, r in enumerate(self.radii):
                base = self.offsets[mi * len(self.radii) + ri]
                blk = flat[base:base + nS * nB * 4 * P].reshape(nS, nB, 4, self.height * M, self.width * M)
                for si, S in enumerate(self.sens):
                    for bi in range(nB):
                        out[(int(M), float(r), int(S), (int(self.bstart[bi]), int(self.blen[bi])))] = blk[si, bi]
        return out

    def squirrel(self, results, fixed_sigma=None, crop=0, device=0):
        """SQUIRREL metrics of every AVG, VAR and TAC2 reconstruction of `results` (run's dict)
        against the INT slice of the same block, as ParametersSweep_ scores its reconstructions
        (gui/ParametersSweep_.java:468-519): {key: {"AVG"|"VAR"|"TAC2": {sigma, alpha, beta,
        rse, rsp}}}, one batched call per magnification."""
        out = {}
        for M in sorted({k[0] for k in results}):
            keys = [k for k in results if k[0] == M]
            sr = np.stack([results[k][c] for k in keys for c in range(3)])
            ref = np.stack([results[k][3] for k in keys])
            m = squirrel(sr, ref, M, fixed_sigma=fixed_sigma, crop=crop,
                         ref_index=[i // 3 for i in range(3 * len(keys))], device=device)
            for i, k in enumerate(keys):
                out[k] = {name: {f: float(m[f][3 * i + c]) for f in ("sigma", "alpha", "beta", "rse", "rsp")}
                          for c, name in enumerate(("AVG", "VAR", "TAC2"))}
        return out

    def run(self, stack, out=None):
        """Runs the sweep on host frames.  ``out``: optional flat float32 array of ``self.total``
        floats to fill (e.g. the numpy view of a pinned torch tensor: a one-device sweep then copies
        each (magnification, radius) pair's outputs out while the next pairs compute)."""
        a = np.asarray(stack)
        if tuple(a.shape) != (self.n_frames, self.height, self.width):
            raise EsrrfError(f"stack must be [{self.n_frames}][{self.height}][{self.width}], got {list(a.shape)}")
        if a.dtype == np.uint16:
            a = np.ascontiguousarray(a)
            is_u16 = 1
        else:
            a = np.ascontiguousarray(a, np.float32)
            is_u16 = 0
        if out is None:
            flat = np.empty(self.total, np.float32)
        else:
            flat = out
            if flat.dtype != np.float32 or flat.size != self.total or not flat.flags.c_contiguous:
                raise EsrrfError("out must be a contiguous float32 array of the sweep's total size")
        _lib.check(self._h, lib().esrrf_sweep_run(self._h, a.ctypes.data_as(ctypes.c_void_p), is_u16,
                                                  flat.ctypes.data_as(ctypes.c_void_p)), sweep=True)
        return self.unpack(flat)

    def release(self):
        if self._h:
            lib().esrrf_sweep_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def rolling(stack, magnification, fwhm, sensitivity, blocks, int_weighting=True,
            interpolation="fht", drift=None, devices=None):
    """Rolling analysis over arbitrary (start, length) blocks, each frame interpolated (or its
    gradients resampled, ``interpolation="bicubic"``) and run through the RGC once:
    {(start, length): [4][HM][WM]}.

    ``drift``: one (shift_x, shift_y) pair of arrays per block, each of the block's length in raw
    pixels -- the per-block arrays the analysis plugin computes relative to each block's first frame
    (gui/LiveSRRF_optimised_.java:283-305).  Blocks that do not overlap run as one sweep with the
    arrays laid end to end; overlapping blocks (a frame with two different shifts) run through the
    engine block by block, as the plugin does.  ``devices``: CUDA ordinals to split the blocks
    across (drift-free or non-overlapping blocks)."""
    a = np.asarray(stack)
    blocks = [(int(st), int(ln)) for st, ln in blocks]
    sweep_drift = None
    if drift is not None:
        if len(drift) != len(blocks):
            raise EsrrfError("drift needs one (shift_x, shift_y) pair per block")
        order = sorted(range(len(blocks)), key=lambda i: blocks[i][0])
        overlap = any(blocks[order[k]][0] + blocks[order[k]][1] > blocks[order[k + 1]][0]
                      for k in range(len(order) - 1))
        if overlap:
            out = {}
            for (st, ln), (dx, dy) in zip(blocks, drift):
                eng = LiveSRRF_CL()
                eng.initialise(a.shape[-1], a.shape[-2], magnification, fwhm, sensitivity, ln, ln,
                               intWeighting=int_weighting, doFHTinterpolation=interpolation == "fht")
                try:
                    eng.resetFramePosition()
                    eng.loadDriftXYGPUbuffer(dx, dy)
                    eng.calculateSRRF(a[st:st + ln])
                    out[(st, ln)] = eng.readSRRFbuffer().copy()
                finally:
                    eng.release()
            return out
        fx = np.zeros(a.shape[0], np.float32)
        fy = np.zeros(a.shape[0], np.float32)
        for (st, ln), (dx, dy) in zip(blocks, drift):
            dx = np.asarray(dx, np.float32).reshape(-1)
            dy = np.asarray(dy, np.float32).reshape(-1)
            if dx.size != ln or dy.size != ln:
                raise EsrrfError("a block's drift arrays must hold one shift per frame of the block")
            fx[st:st + ln] = dx
            fy[st:st + ln] = dy
        sweep_drift = (fx, fy)
    sw = Sweep(a.shape[-1], a.shape[-2], a.shape[0], [magnification], [fwhm], [sensitivity],
               blocks, int_weighting, interpolation=interpolation, drift=sweep_drift, devices=devices)
    try:
        res = sw.run(a)
        return {k[3]: v.copy() for k, v in res.items()}
    finally:
        sw.release()


def squirrel(sr, ref, magnification, fixed_sigma=None, crop=0, error_maps=False, ref_index=None,
             device=0):
    """SQUIRREL metrics (esrrf_squirrel; ErrorMapLiveSRRF.optimise + calculateErrorMap,
    ErrorMapLiveSRRF.java:81-193) of super-resolved images against references.

    sr: [n][H][W]; ref: [n][H][W], [H][W] (one reference for all) or, with ref_index ([n] ints),
    [m][H][W] with image i scored against ref[ref_index[i]]; numpy arrays or torch CUDA tensors.
    fixed_sigma (input pixels) skips the sigma search; crop: border in input pixels.  Returns a
    dict of numpy arrays sigma, alpha, beta, rse, rsp ([n]) and, with error_maps, "error_map"
    [n][H'][W'] (the cropped size)."""
    import torch

    from ._lib import EsrrfSquirrelParams

    dev = f"cuda:{device}"
    srt = torch.as_tensor(sr, dtype=torch.float32, device=dev).contiguous()
    if srt.dim() == 2:
        srt = srt[None]
    reft = torch.as_tensor(ref, dtype=torch.float32, device=dev).contiguous()
    if reft.dim() == 2:
        reft = reft[None]
    n, H, W = srt.shape
    if ref_index is None:
        if reft.shape[0] not in (1, n):
            raise EsrrfError("ref must be [H][W] or [n][H][W] like sr (or give ref_index)")
        ref_index = [i if reft.shape[0] == n else 0 for i in range(n)]
    ref_index = [int(r) for r in ref_index]
    if reft.shape[-2:] != (H, W) or len(ref_index) != n or min(ref_index) < 0 or max(ref_index) >= reft.shape[0]:
        raise EsrrfError("ref images must match sr in size and ref_index must select them")
    both = torch.cat([srt.reshape(-1), reft.reshape(-1)])
    P = H * W
    sro = (ctypes.c_size_t * n)(*[i * P for i in range(n)])
    rfo = (ctypes.c_size_t * n)(*[n * P + r * P for r in ref_index])
    cb = int(crop) * int(magnification) if crop else 0
    maps = torch.empty((n, H - 2 * cb, W - 2 * cb), dtype=torch.float32, device=dev) if error_maps else None
    out = {k: np.empty(n, np.float32) for k in ("sigma", "alpha", "beta", "rse", "rsp")}
    fp = ctypes.POINTER(ctypes.c_float)
    p = EsrrfSquirrelParams(W, H, int(magnification), int(fixed_sigma is not None),
                            float(fixed_sigma or 0.0), int(crop),
                            ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream))
    with torch.cuda.device(device):
        _lib.check(None, lib().esrrf_squirrel(ctypes.byref(p), n, ctypes.c_void_p(both.data_ptr()), sro, rfo,
                                              *[out[k].ctypes.data_as(fp) for k in ("sigma", "alpha", "beta", "rse", "rsp")],
                                              ctypes.c_void_p(maps.data_ptr()) if maps is not None else None),
                   squirrel=True)
    if maps is not None:
        out["error_map"] = maps.cpu().numpy()
    return out


def frc_size(width, height):
    """(padded size N, number of rings N/2 + 1) of esrrf_frc for images of this size."""
    N, R = ctypes.c_int(), ctypes.c_int()
    _lib.check(None, lib().esrrf_frc_size(int(width), int(height), ctypes.byref(N), ctypes.byref(R)),
               frc=True)
    return N.value, R.value


def frc(a, b, pixel_size=1.0, curves=False, device=0):
    """FIRE resolution (esrrf_frc) of image pairs: a, b [n][H][W] or [H][W], numpy or torch CUDA.
    Returns float32 [n] in pixel_size units (NaN: no 1/7 crossing), with curves also the FRC
    curves [n][N/2 + 1]."""
    import torch

    from ._lib import EsrrfFrcParams

    dev = f"cuda:{device}"
    at = torch.as_tensor(a, dtype=torch.float32, device=dev).contiguous()
    bt = torch.as_tensor(b, dtype=torch.float32, device=dev).contiguous()
    if at.dim() == 2:
        at, bt = at[None], bt[None]
    if at.shape != bt.shape:
        raise EsrrfError("frc: the two image stacks differ in shape")
    n, H, W = at.shape
    _, R = frc_size(W, H)
    both = torch.cat([at.reshape(-1), bt.reshape(-1)])
    P = H * W
    ao = (ctypes.c_size_t * n)(*[i * P for i in range(n)])
    bo = (ctypes.c_size_t * n)(*[(n + i) * P for i in range(n)])
    fire = np.empty(n, np.float32)
    cv = np.empty((n, R), np.float32) if curves else None
    fp = ctypes.POINTER(ctypes.c_float)
    p = EsrrfFrcParams(W, H, float(pixel_size), ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream))
    with torch.cuda.device(device):
        _lib.check(None, lib().esrrf_frc(ctypes.byref(p), n, ctypes.c_void_p(both.data_ptr()), ao, bo,
                                         fire.ctypes.data_as(fp), cv.ctypes.data_as(fp) if cv is not None else None),
                   frc=True)
    return (fire, cv) if curves else fire


def sweep_frc(stack, magnifications, radii, sensitivities, n_frames, pixel_size=1.0, int_weighting=True,
              device=0):
    """The sweep's FRC mode (gui/ParametersSweep_.java:403-447): every (M, radius, S) reconstructed
    from the odd frames (1, 3, 5, ... in ImageJ's 1-based numbering) and from the even frames of the
    first 2 n_frames, and the FIRE resolution of each AVG, VAR and TAC2 pair in units of
    pixel_size / M (the raw pixel size divided by the magnification, as the reference's output
    calibration).  Returns ({(M, radius, S): {"AVG"|"VAR"|"TAC2": resolution}}, odd results, even
    results); like the reference, the even-frame reconstructions are the sweep's images."""
    a = np.asarray(stack)
    if a.shape[0] < 2 * int(n_frames):
        raise EsrrfError(f"FRC mode needs {2 * int(n_frames)} frames, the stack has {a.shape[0]}")
    halves = []
    for start in (0, 1):
        sub = np.ascontiguousarray(a[start:2 * int(n_frames):2])
        sw = Sweep(a.shape[-1], a.shape[-2], sub.shape[0], magnifications, radii, sensitivities,
                   [(0, sub.shape[0])], int_weighting=int_weighting, device=device)
        try:
            halves.append({k[:3]: v.copy() for k, v in sw.run(sub).items()})
        finally:
            sw.release()
    odd, even = halves
    out = {}
    for M in sorted({k[0] for k in odd}):
        keys = [k for k in odd if k[0] == M]
        A = np.stack([odd[k][c] for k in keys for c in range(3)])
        B = np.stack([even[k][c] for k in keys for c in range(3)])
        res = frc(A, B, pixel_size=float(pixel_size) / M, device=device)
        for i, k in enumerate(keys):
            out[k] = {name: float(res[3 * i + c]) for c, name in enumerate(("AVG", "VAR", "TAC2"))}
    return out, odd, even


def _device_frames(frames, device):
    """[T][H][W] frames on cuda:device as (tensor, is_u16); uint16 travels as its int16 bit pattern."""
    import torch

    dev = f"cuda:{device}"
    if isinstance(frames, torch.Tensor):
        t = frames
        if t.dtype in (torch.int16, torch.uint16):
            return t.to(dev).view(torch.int16).contiguous(), 1
        return t.to(device=dev, dtype=torch.float32).contiguous(), 0
    a = np.ascontiguousarray(frames)
    if a.dtype == np.uint16:
        return torch.from_numpy(a.view(np.int16)).to(dev), 1
    return torch.from_numpy(a.astype(np.float32, copy=False)).to(dev), 0


def drift_window(width, height, max_shift=None) -> int:
    """Lag radius R that estimate_drift searches (esrrf_drift_window)."""
    R = ctypes.c_int()
    _lib.check(None, lib().esrrf_drift_window(int(width), int(height), int(max_shift or 0), ctypes.byref(R)),
               drift=True)
    return R.value


def estimate_drift(frames, ref_frame=0, max_shift=None, return_map=False, device=0):
    """Drift of every frame relative to frames[ref_frame] (esrrf_estimate_drift; the restatement of
    XYShiftCalculator.calculateShiftArray, XYShiftCalculator.java:26-48).

    frames: [T][H][W] uint16 or float32, numpy or torch.  Returns (shift_x, shift_y) float32 [T], the
    displacement of each frame's content relative to the reference frame (what
    LiveSRRF_CL.loadDriftXYGPUbuffer takes); with return_map also the cross-correlation maps
    [T][2R+1][2R+1] (lag (sy, sx) at [sy + R][sx + R])."""
    import torch

    t, is_u16 = _device_frames(frames, device)
    if t.dim() == 2:
        t = t[None]
    n, H, W = t.shape
    R = drift_window(W, H, max_shift)
    sx = np.empty(n, np.float32)
    sy = np.empty(n, np.float32)
    ccm = torch.empty((n, 2 * R + 1, 2 * R + 1), dtype=torch.float32, device=t.device) if return_map else None
    fp = ctypes.POINTER(ctypes.c_float)
    with torch.cuda.device(device):
        _lib.check(None, lib().esrrf_estimate_drift(
            ctypes.c_void_p(t.data_ptr()), is_u16, n, W, H, int(ref_frame), int(max_shift or 0),
            sx.ctypes.data_as(fp), sy.ctypes.data_as(fp),
            ctypes.c_void_p(ccm.data_ptr()) if ccm is not None else None,
            ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)), drift=True)
    if return_map:
        return sx, sy, ccm.cpu().numpy()
    return sx, sy


class XYShiftCalculator:
    """Mirror of nanoj.liveSRRF.XYShiftCalculator (XYShiftCalculator.java:12-48) on the GPU.

    calculateShiftArray(indexStart, nFrameForSRRF) takes the 1-based stack index of the block's
    first frame (the reference frame, as ImageJ's getProcessor does) and fills shiftX and shiftY
    for the nFrameForSRRF frames from there."""

    def __init__(self, imp, prof=None, max_shift=None, device=0):
        self.ims = imp
        self.max_shift = max_shift
        self.device = device
        self.shiftX = None
        self.shiftY = None

    def calculateShiftArray(self, indexStart, nFrameForSRRF):
        i0 = int(indexStart) - 1
        if i0 < 0 or i0 + int(nFrameForSRRF) > len(self.ims):
            raise EsrrfError("indexStart/nFrameForSRRF outside the stack")
        self.shiftX, self.shiftY = estimate_drift(self.ims[i0:i0 + int(nFrameForSRRF)], 0, self.max_shift,
                                                  device=self.device)


class Adjoint:
    """Differentiable eSRRF (esrrf_adjoint_*, esrrf_loss_and_grad): a re-blur fidelity loss of the
    2-D FHT-path AVG reconstruction and its gradients w.r.t. radius, a real sensitivity, the
    re-blur sigma and every input pixel.  Frames are passed as a torch CUDA tensor (float32,
    [T][h][w]) or a numpy array (copied to the device)."""

    def __init__(self, width, height, n_frames, magnification, device=0):
        h = ctypes.c_void_p()
        _lib.check(None, lib().esrrf_adjoint_create(int(width), int(height), int(n_frames),
                                                    int(magnification), int(device), ctypes.byref(h)),
                   adjoint=True)
        self._h = h
        self.shape = (int(n_frames), int(height), int(width))
        self.device = int(device)

    def _dev(self, frames):
        import torch

        if isinstance(frames, torch.Tensor):
            t = frames.to(device=f"cuda:{self.device}", dtype=torch.float32).contiguous()
        else:
            t = torch.from_numpy(np.ascontiguousarray(frames, np.float32)).to(f"cuda:{self.device}")
        if tuple(t.shape) != self.shape:
            raise EsrrfError(f"frames must be {list(self.shape)}, got {list(t.shape)}")
        return t

    def loss(self, frames, fwhm, sensitivity, sigma):
        t = self._dev(frames)
        L = ctypes.c_double()
        _lib.check(self._h, lib().esrrf_adjoint_forward(self._h, ctypes.c_void_p(t.data_ptr()),
                                                        float(fwhm), float(sensitivity), float(sigma),
                                                        ctypes.byref(L)), adjoint=True)
        return L.value

    def loss_and_grad(self, frames, fwhm, sensitivity, sigma, pixel_grad=True):
        """(loss, {"fwhm", "S", "sigma"}, d loss / d frames as a torch tensor or None)."""
        import torch

        t = self._dev(frames)
        L = ctypes.c_double()
        g = (ctypes.c_double * 3)()
        gf = torch.empty_like(t) if pixel_grad else None
        _lib.check(self._h, lib().esrrf_loss_and_grad(
            self._h, ctypes.c_void_p(t.data_ptr()), float(fwhm), float(sensitivity), float(sigma),
            ctypes.byref(L), g, ctypes.c_void_p(gf.data_ptr() if gf is not None else None)), adjoint=True)
        return L.value, {"fwhm": g[0], "S": g[1], "sigma": g[2]}, gf

    def release(self):
        if self._h:
            lib().esrrf_adjoint_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def gradient_search(adj, frames, fwhm0, sens0, sigma0, steps=40, lr=(0.05, 0.1, 0.05),
                    bounds=((0.5, 3.0), (0.5, 6.0), (0.5, 8.0))):
    """Projected gradient descent with a backtracking step on (radius, sensitivity, re-blur
    sigma), the search that stands beside the grid sweep.  Returns the trajectory."""
    x = np.array([fwhm0, sens0, sigma0], np.float64)
    lo = np.array([b[0] for b in bounds])
    hi = np.array([b[1] for b in bounds])
    step = np.array(lr, np.float64)
    L, g, _ = adj.loss_and_grad(frames, *x, pixel_grad=False)
    traj = [(x.copy(), L)]
    for _ in range(steps):
        gv = np.array([g["fwhm"], g["S"], g["sigma"]])
        scale = np.abs(gv).max() or 1.0
        accepted = False
        for _ in range(8):
            xn = np.clip(x - step * gv / scale, lo, hi)
            Ln = adj.loss(frames, *xn)
            if Ln < L:
                accepted = True
                break
            step = step * 0.5
        if not accepted:
            break
        x = xn
        L, g, _ = adj.loss_and_grad(frames, *x, pixel_grad=False)
        step = step * 1.5
        traj.append((x.copy(), L))
    return traj
