"""GPU test of esrrf_fht_block_noalloc, the entry point for callers that cannot allocate device
memory when they reconstruct (e.g. a live-acquisition callback, where cudaMalloc could stall
the camera stream by synchronising the device).  It must give the same block as the regular
handle-based entry points and the oracle, on two calls in a row (the shared static scratch keeps
the previous call's contents, so the second call checks that everything that must start at zero
is cleared), allocate no device memory, and reject frame sizes beyond its 64 MiB scratch with a
clear error.

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


def _noalloc(L, d_frames, n, w, h, M, fwhm, S, d_out, stream):
    err = ctypes.create_string_buffer(512)
    rc = L.esrrf_fht_block_noalloc(ctypes.c_void_p(d_frames.data_ptr()), 1, n, w, h, M, ctypes.c_float(fwhm), S,
                                   1, ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream), err, len(err))
    assert rc == 0, err.value.decode()


def test_noalloc_matches_oracle_and_reuses_its_tables(esrrf_mod, oracle_mod):
    """Against the oracle's block (the C restatement, pinned to the reference kernels), for a
    small frame whose launches split into frame groups; a repeated call with the same key reuses
    the tables kept in the array and gives the identical result."""
    import torch

    from esrrf import synth

    L = esrrf_mod.lib()
    n, h, w, M, fwhm, S = 12, 24, 40, 4, 1.5, 2
    raw = synth.small_stack(33, n, h, w, emitters=10)
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw.astype(np.float32), M), M, fwhm, S)
    d_frames = torch.from_numpy(raw.view(np.int16)).cuda()
    outs = []
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        d_out = torch.full((4, h * M, w * M), float("nan"), dtype=torch.float32, device="cuda")
        _noalloc(L, d_frames, n, w, h, M, fwhm, S, d_out, stream)
        torch.cuda.synchronize()
        outs.append(d_out.cpu().numpy())
    for k in range(4):
        assert rel_err(outs[0][k], ref[k]) < TOL, (k, rel_err(outs[0][k], ref[k]))
    np.testing.assert_array_equal(outs[0], outs[1])


def test_noalloc_allocates_no_device_memory(esrrf_mod):
    """The entry point's defining property: once its kernels are loaded (warm-up calls at both
    frame sizes), a call with a changed frame size -- which rebuilds the tables in the array -- and
    a repeated call leave the device's free memory unchanged."""
    import torch

    from esrrf import synth

    L = esrrf_mod.lib()
    M, fwhm, S = 4, 1.5, 2
    sizes = [(48, 56), (64, 64), (48, 56), (48, 56)]
    ins = [torch.from_numpy(synth.small_stack(40 + i, 6, h, w).view(np.int16)).cuda()
           for i, (w, h) in enumerate(sizes)]
    outs = [torch.empty((4, h * M, w * M), dtype=torch.float32, device="cuda") for w, h in sizes]
    stream = torch.cuda.current_stream().cuda_stream
    for i in (0, 1):
        _noalloc(L, ins[i], 6, *sizes[i], M, fwhm, S, outs[i], stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for i in (2, 3):
        _noalloc(L, ins[i], 6, *sizes[i], M, fwhm, S, outs[i], stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.isfinite(outs[3]).all()


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
    # a magnified side beyond 2^20 pixels is rejected before any size arithmetic
    rc = L.esrrf_fht_block_noalloc(ctypes.c_void_p(d_frames.data_ptr()), 1, 2, 1 << 17, 8, 16,
                                   ctypes.c_float(1.5), 2, 1, ctypes.c_void_p(d_out.data_ptr()),
                                   None, err, len(err))
    assert rc == -1 and b"1048576" in err.value
