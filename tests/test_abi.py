"""CPU tests of the C ABI: the library loads, exports every symbol include/esrrf.h declares,
and the ctypes view of esrrf_params matches the C layout.  No GPU work is done."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "esrrf.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(esrrf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(esrrf_mod):
    from esrrf import _lib
    L = esrrf_mod.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


@pytest.mark.parametrize("py_name,c_name", [("EsrrfParams", "esrrf_params"),
                                             ("EsrrfSweepParams", "esrrf_sweep_params"),
                                             ("EsrrfSquirrelParams", "esrrf_squirrel_params"),
                                             ("EsrrfFrcParams", "esrrf_frc_params")])
def test_params_layout_matches_c(py_name, c_name):
    from esrrf import _lib
    EsrrfParams = getattr(_lib, py_name)
    fields = [f for f, _ in EsrrfParams._fields_]
    prog = "#include <stdio.h>\n#include <stddef.h>\n#include \"esrrf.h\"\nint main(){"
    prog += f'printf("%zu\\n", sizeof({c_name}));'
    for f in fields:
        prog += f'printf("%zu\\n", offsetof({c_name}, {f}));'
    prog += "return 0;}"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        vals = [int(x) for x in subprocess.run([exe], capture_output=True, text=True,
                                               check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(EsrrfParams)
    for f, off in zip(fields, vals[1:]):
        assert getattr(EsrrfParams, f).offset == off, f


def test_version_and_defaults(esrrf_mod):
    L = esrrf_mod.lib()
    assert L.esrrf_get_version().decode().startswith("0.")
    p = esrrf_mod.default_params()
    # reference GUI defaults (gui/LiveSRRF_optimised_.java:128-134)
    assert (p.magnification, p.sensitivity, p.n_frame_for_srrf, p.block_length) == (5, 1, 100, 20000)
    assert abs(p.fwhm - 2.0) < 1e-6 and p.int_weighting == 1 and p.interp == 0


def test_invalid_parameters_are_rejected_before_device_work(esrrf_mod):
    """Parameter validation runs on the host and reports through esrrf_last_error(NULL)."""
    L = esrrf_mod.lib()
    p = esrrf_mod.default_params()
    p.width, p.height = 2, 64
    h = ctypes.c_void_p()
    rc = L.esrrf_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == -1 and not h.value
    assert b"width" in L.esrrf_last_error(None)
    p.width, p.height, p.magnification = 64, 64, 0
    assert L.esrrf_create(ctypes.byref(p), ctypes.byref(h)) == -1
    p.magnification, p.n_frame_for_srrf = 4, 0
    assert L.esrrf_create(ctypes.byref(p), ctypes.byref(h)) == -1
    p.n_frame_for_srrf, p.n_planes = 10, 3  # 3-D without calibration arrays
    assert L.esrrf_create(ctypes.byref(p), ctypes.byref(h)) == -1
    p.n_planes, p.width, p.height, p.magnification = 0, 12000, 12000, 4  # 48000^2 output pixels
    assert L.esrrf_create(ctypes.byref(p), ctypes.byref(h)) == -1
    assert b"too large" in L.esrrf_last_error(None)


def test_null_handles_are_rejected(esrrf_mod):
    L = esrrf_mod.lib()
    assert L.esrrf_destroy(None) == -1
    assert L.esrrf_reset_frame_position(None) == -1
    assert L.esrrf_read_srrf(None, None) == -1
    assert L.esrrf_request_cancel(None) == -1
    # the bounded-wait diagnostic checks its limit before any device work
    assert L.esrrf_check_bounded_wait(0, 0, 0) == -1
    assert L.esrrf_check_bounded_wait(0, 0, 2_000_000_000) == -1


def test_no_cpu_fallback_without_library(monkeypatch):
    """The package fails loudly when the CUDA library is missing."""
    from esrrf import _lib
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libesrrf.so")
    with pytest.raises(_lib.EsrrfError):
        _lib.lib()


def test_drift_window_matches_oracle(esrrf_mod):
    """esrrf_drift_window is host arithmetic only (no device work): same lag radius as the oracle."""
    from oracle import drift_oracle as D
    for w, h, ms in [(512, 512, None), (20, 17, None), (200, 180, 80), (200, 180, 500), (3, 3, None)]:
        assert esrrf_mod.drift_window(w, h, ms) == D.window(w, h, ms)
    with pytest.raises(esrrf_mod.EsrrfError):
        esrrf_mod.drift_window(2, 64)


def test_sweep_rejects_bad_parameters_before_any_device_work(esrrf_mod):
    """esrrf_sweep_create validates its parameters first (no GPU needed): an unknown
    interpolation, a block outside the stack, an empty radius list."""
    from esrrf import _lib
    ip = ctypes.POINTER(ctypes.c_int)
    fp = ctypes.POINTER(ctypes.c_float)
    mags = (ctypes.c_int * 1)(2)
    radii = (ctypes.c_float * 1)(1.5)
    sens = (ctypes.c_int * 1)(1)
    bs = (ctypes.c_int * 1)(0)

    def create(interp=0, blen=10, n_radius=1):
        bl = (ctypes.c_int * 1)(blen)
        p = _lib.EsrrfSweepParams(32, 32, 10, 1, ctypes.cast(mags, ip), n_radius, ctypes.cast(radii, fp),
                                  1, ctypes.cast(sens, ip), 1, ctypes.cast(bs, ip), ctypes.cast(bl, ip),
                                  1, -1, interp)
        h = ctypes.c_void_p()
        rc = esrrf_mod.lib().esrrf_sweep_create(ctypes.byref(p), ctypes.byref(h))
        return rc, esrrf_mod.lib().esrrf_sweep_last_error(None).decode()

    invalid = -1  # ESRRF_ERR_INVALID
    rc, msg = create(interp=7)
    assert rc == invalid and "interpolation" in msg
    rc, msg = create(blen=11)
    assert rc == invalid and "outside the stack" in msg
    rc, msg = create(n_radius=0)
    assert rc == invalid and "non-empty" in msg
    mags[0] = 16
    p = _lib.EsrrfSweepParams(4000, 4000, 10, 1, ctypes.cast(mags, ip), 1, ctypes.cast(radii, fp), 1,
                              ctypes.cast(sens, ip), 1, ctypes.cast(bs, ip), ctypes.cast((ctypes.c_int * 1)(10), ip),
                              1, -1, 0)
    h = ctypes.c_void_p()
    assert esrrf_mod.lib().esrrf_sweep_create(ctypes.byref(p), ctypes.byref(h)) == invalid
    assert "too large" in esrrf_mod.lib().esrrf_sweep_last_error(None).decode()
