"""GPU test of esrrf_fht_block_noalloc, the entry point for callers that cannot allocate device
memory when they reconstruct (e.g. a live-acquisition callback, where cudaMalloc could stall
the camera stream by synchronising the device).  It must give the same block as the regular
handle-based entry points, on two calls in a row (the shared static scratch keeps the previous
call's contents, so the second call checks that everything that must start at zero is cleared),
and reject frame sizes beyond its 64 MiB scratch with a clear error.

Kept in its own file, collected last, so a run that stops at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _existing_entry_point(esrrf, L, d_frames, n, w, h, M, fwhm, S, d_out):
    eng = esrrf.LiveSRRF_CL()
    eng.initialise(w, h, M, fwhm, S, n, n)
    try:
        H = eng.handle
        esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
        esrrf._lib.check(H, L.esrrf_calculate_srrf_u16_device(H, ctypes.c_void_p(d_frames), n))
        esrrf._lib.check(H, L.esrrf_read_srrf_device(H, ctypes.c_void_p(d_out)))
    finally:
        eng.release()


def test_noalloc_matches_handle_entry_points_twice(esrrf_mod):
    import torch

    from esrrf import synth

    L = esrrf_mod.lib()
    n, h, w, M, fwhm, S = 10, 64, 64, 4, 1.5, 2
    stacks = [synth.small_stack(31, n, h, w, emitters=20), synth.small_stack(32, n, h, w, emitters=6)]
    stream = torch.cuda.current_stream()
    err = ctypes.create_string_buffer(512)
    for raw in stacks:
        d_frames = torch.from_numpy(raw.view(np.int16)).cuda()
        d_ref = torch.empty((4, h * M, w * M), dtype=torch.float32, device="cuda")
        d_new = torch.full((4, h * M, w * M), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        _existing_entry_point(esrrf_mod, L, d_frames.data_ptr(), n, w, h, M, fwhm, S,
                              d_ref.data_ptr())
        rc = L.esrrf_fht_block_noalloc(ctypes.c_void_p(d_frames.data_ptr()), 1, n, w, h, M,
                                       ctypes.c_float(fwhm), S, 1, ctypes.c_void_p(d_new.data_ptr()),
                                       ctypes.c_void_p(stream.cuda_stream), err, len(err))
        assert rc == 0, err.value.decode()
        torch.cuda.synchronize()
        ref = d_ref.cpu().numpy()
        got = d_new.cpu().numpy()
        assert np.isfinite(got).all()
        for k in range(4):
            assert rel_err(got[k], ref[k]) < TOL, (k, rel_err(got[k], ref[k]))


def test_noalloc_rejects_sizes_beyond_its_scratch(esrrf_mod):
    import torch

    L = esrrf_mod.lib()
    err = ctypes.create_string_buffer(512)
    d_frames = torch.zeros((2, 512, 512), dtype=torch.int16, device="cuda")
    d_out = torch.empty((4, 16, 16), dtype=torch.float32, device="cuda")  # never written
    rc = L.esrrf_fht_block_noalloc(ctypes.c_void_p(d_frames.data_ptr()), 1, 2, 512, 512, 4,
                                   ctypes.c_float(1.5), 2, 1, ctypes.c_void_p(d_out.data_ptr()),
                                   None, err, len(err))
    assert rc == -1
    assert b"MiB" in err.value
