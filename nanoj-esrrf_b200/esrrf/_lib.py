"""ctypes binding of include/esrrf.h (libesrrf.so, built in-tree under nanoj-esrrf_b200/lib/)."""
from __future__ import annotations

import ctypes
import os

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libesrrf.so")

_f32p = ctypes.POINTER(ctypes.c_float)


class EsrrfParams(ctypes.Structure):
    """esrrf_params (include/esrrf.h)."""

    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("magnification", ctypes.c_int),
        ("fwhm", ctypes.c_float),
        ("sensitivity", ctypes.c_int),
        ("n_frames_on_gpu", ctypes.c_int),
        ("n_frame_for_srrf", ctypes.c_int),
        ("block_length", ctypes.c_int),
        ("device", ctypes.c_int),
        ("int_weighting", ctypes.c_int),
        ("mp_correction", ctypes.c_int),
        ("interp", ctypes.c_int),
        ("fht_scale", ctypes.c_int),
        ("kernel", ctypes.c_int),
        ("frames_per_launch", ctypes.c_int),
        ("n_planes", ctypes.c_int),
        ("roi", _f32p), ("theta_deg", _f32p), ("shift_x", _f32p), ("shift_y", _f32p),
        ("intensity_coeff", _f32p),
        ("background", ctypes.c_float),
        ("axial_offset_nm", ctypes.c_float),
        ("pixel_size_um", ctypes.c_float),
    ]


class EsrrfError(RuntimeError):
    pass


STATUS = {0: "OK", 1: "CANCELLED", -1: "INVALID", -2: "CUDA", -3: "NOMEM", -4: "STATE",
          -5: "TIMEOUT", -6: "NODEVICE"}

# Every symbol the header declares, with its ctypes signature.
_c = ctypes
SIGNATURES = {
    "esrrf_get_version": (_c.c_char_p, []),
    "esrrf_device_count": (_c.c_int, [_c.POINTER(_c.c_int)]),
    "esrrf_device_info": (_c.c_int, [_c.c_int, _c.c_char_p, _c.c_size_t, _c.POINTER(_c.c_int),
                                     _c.POINTER(_c.c_int)]),
    "esrrf_default_params": (None, [_c.POINTER(EsrrfParams)]),
    "esrrf_create": (_c.c_int, [_c.POINTER(EsrrfParams), _c.POINTER(_c.c_void_p)]),
    "esrrf_destroy": (_c.c_int, [_c.c_void_p]),
    "esrrf_set_drift": (_c.c_int, [_c.c_void_p, _f32p, _f32p, _c.c_int]),
    "esrrf_reset_frame_position": (_c.c_int, [_c.c_void_p]),
    "esrrf_calculate_srrf_u16": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int]),
    "esrrf_calculate_srrf_f32": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int]),
    "esrrf_calculate_srrf_u16_device": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int]),
    "esrrf_calculate_srrf_f32_device": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int]),
    "esrrf_read_srrf": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "esrrf_read_srrf_async": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "esrrf_frames_per_launch": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_int)]),
    "esrrf_read_aligned_pixels": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_size_t]),
    "esrrf_read_mp_maps": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_size_t]),
    "esrrf_read_srrf_device": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "esrrf_output_shape": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_int), _c.POINTER(_c.c_int),
                                      _c.POINTER(_c.c_int)]),
    "esrrf_read_gradients": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_size_t]),
    "esrrf_finish_queue": (_c.c_int, [_c.c_void_p]),
    "esrrf_request_cancel": (_c.c_int, [_c.c_void_p]),
    "esrrf_check_bounded_wait": (_c.c_int, [_c.c_int, _c.c_int, _c.c_longlong]),
    "esrrf_last_error": (_c.c_char_p, [_c.c_void_p]),
    "esrrf_set_timing": (_c.c_int, [_c.c_void_p, _c.c_int]),
    "esrrf_set_stream": (_c.c_int, [_c.c_void_p, _c.c_void_p]),
    "esrrf_last_timing": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_float), _c.POINTER(_c.c_float),
                                     _c.POINTER(_c.c_int)]),
    "esrrf_fht_block_noalloc": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_int, _c.c_int, _c.c_int,
                                           _c.c_int, _c.c_float, _c.c_int, _c.c_int, _c.c_void_p,
                                           _c.c_void_p, _c.c_char_p, _c.c_size_t]),
}


class EsrrfSweepParams(ctypes.Structure):
    """esrrf_sweep_params (include/esrrf.h)."""

    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("n_frames", ctypes.c_int),
        ("n_mag", ctypes.c_int), ("magnifications", ctypes.POINTER(ctypes.c_int)),
        ("n_radius", ctypes.c_int), ("radii", _f32p),
        ("n_sens", ctypes.c_int), ("sensitivities", ctypes.POINTER(ctypes.c_int)),
        ("n_blocks", ctypes.c_int), ("block_start", ctypes.POINTER(ctypes.c_int)),
        ("block_length", ctypes.POINTER(ctypes.c_int)),
        ("int_weighting", ctypes.c_int), ("device", ctypes.c_int), ("interp", ctypes.c_int),
        ("drift_x", _f32p), ("drift_y", _f32p),
        ("n_devices", ctypes.c_int), ("devices", ctypes.POINTER(ctypes.c_int)),
    ]


class EsrrfSquirrelParams(ctypes.Structure):
    """esrrf_squirrel_params (include/esrrf.h)."""

    _fields_ = [
        ("width", ctypes.c_int), ("height", ctypes.c_int), ("magnification", ctypes.c_int),
        ("fix_sigma", ctypes.c_int), ("fixed_sigma", ctypes.c_float), ("crop", ctypes.c_int),
        ("stream", ctypes.c_void_p),
    ]


class EsrrfFrcParams(ctypes.Structure):
    """esrrf_frc_params (include/esrrf.h)."""

    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("pixel_size", ctypes.c_float),
                ("stream", ctypes.c_void_p)]


SIGNATURES.update({
    "esrrf_squirrel": (_c.c_int, [_c.POINTER(EsrrfSquirrelParams), _c.c_int, _c.c_void_p,
                                  _c.POINTER(_c.c_size_t), _c.POINTER(_c.c_size_t), _f32p, _f32p,
                                  _f32p, _f32p, _f32p, _c.c_void_p]),
    "esrrf_squirrel_last_error": (_c.c_char_p, []),
    "esrrf_drift_window": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.POINTER(_c.c_int)]),
    "esrrf_estimate_drift": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_int,
                                        _c.c_int, _f32p, _f32p, _c.c_void_p, _c.c_void_p]),
    "esrrf_drift_last_error": (_c.c_char_p, []),
    "esrrf_frc_size": (_c.c_int, [_c.c_int, _c.c_int, _c.POINTER(_c.c_int), _c.POINTER(_c.c_int)]),
    "esrrf_frc": (_c.c_int, [_c.c_void_p, _c.c_int, _c.c_void_p, _c.POINTER(_c.c_size_t),
                             _c.POINTER(_c.c_size_t), _f32p, _f32p]),
    "esrrf_frc_last_error": (_c.c_char_p, []),
})

SIGNATURES.update({
    "esrrf_sweep_create": (_c.c_int, [_c.POINTER(EsrrfSweepParams), _c.POINTER(_c.c_void_p)]),
    "esrrf_sweep_output_layout": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_size_t),
                                             _c.POINTER(_c.c_size_t)]),
    "esrrf_sweep_run_device": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int, _c.c_void_p]),
    "esrrf_sweep_run": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_int, _c.c_void_p]),
    "esrrf_sweep_launch_count": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_int)]),
    "esrrf_sweep_shard_count": (_c.c_int, [_c.c_void_p, _c.POINTER(_c.c_int)]),
    "esrrf_tune_report": (_c.c_int, [_c.c_void_p, _c.c_char_p, _c.c_size_t]),
    "esrrf_sweep_plan": (_c.c_int, [_c.POINTER(EsrrfSweepParams), _c.POINTER(_c.c_int),
                                    _c.POINTER(_c.c_int), _c.POINTER(_c.c_double)]),
    "esrrf_sweep_last_error": (_c.c_char_p, [_c.c_void_p]),
    "esrrf_sweep_destroy": (_c.c_int, [_c.c_void_p]),
    "esrrf_adjoint_create": (_c.c_int, [_c.c_int, _c.c_int, _c.c_int, _c.c_int, _c.c_int,
                                        _c.POINTER(_c.c_void_p)]),
    "esrrf_adjoint_forward": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_float, _c.c_float,
                                         _c.c_float, _c.POINTER(_c.c_double)]),
    "esrrf_loss_and_grad": (_c.c_int, [_c.c_void_p, _c.c_void_p, _c.c_float, _c.c_float, _c.c_float,
                                       _c.POINTER(_c.c_double), _c.POINTER(_c.c_double), _c.c_void_p]),
    "esrrf_adjoint_last_error": (_c.c_char_p, [_c.c_void_p]),
    "esrrf_adjoint_destroy": (_c.c_int, [_c.c_void_p]),
})

_LIB = None


def lib():
    """Load libesrrf.so; raises if it has not been built (there is no fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise EsrrfError(f"libesrrf.so not built ({LIB_PATH}); run nanoj-esrrf_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(handle, rc: int, sweep: bool = False, adjoint: bool = False, squirrel: bool = False,
          drift: bool = False, frc: bool = False) -> None:
    if rc == 0:
        return
    if squirrel or drift or frc:
        msg = (lib().esrrf_drift_last_error if drift else
               lib().esrrf_frc_last_error if frc else lib().esrrf_squirrel_last_error)()
        msg = msg.decode() if msg else ""
        raise EsrrfError(f"esrrf status {STATUS.get(rc, rc)}: {msg}")
    fn = lib().esrrf_adjoint_last_error if adjoint else (
        lib().esrrf_sweep_last_error if sweep else lib().esrrf_last_error)
    msg = fn(handle)
    msg = msg.decode() if msg else ""
    raise EsrrfError(f"esrrf status {STATUS.get(rc, rc)}: {msg}")
