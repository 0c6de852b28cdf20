"""Queued read-back (esrrf_read_srrf_async + finishQueue) and pushes that return before their
kernels finish: the same blocks as synchronous reads, bit for bit, with pinned and pageable host
frames, one chunk per push (staging buffers reused across calls), more reads queued than slots."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def blocks_sync(esrrf, stack, M, nf, push):
    eng = esrrf.LiveSRRF_CL()
    eng.initialise(stack.shape[-1], stack.shape[-2], M, 1.5, 2, nf, nf, framesPerLaunch=4)
    out = []
    try:
        for b in range(stack.shape[0] // nf):
            eng.resetFramePosition()
            for s in range(0, nf, push):
                assert not eng.calculateSRRF(stack[b * nf + s:b * nf + s + push])
            out.append(eng.readSRRFbuffer().copy())
    finally:
        eng.release()
    return out


@pytest.mark.parametrize("pinned", [False, True])
def test_async_reads_match_sync(esrrf_mod, pinned):
    import torch
    from esrrf import synth
    stack = synth.small_stack(3, 40, 96, 80)  # 5 blocks of 8 frames, 4 frames per launch
    M, nf, push = 3, 8, 4
    want = blocks_sync(esrrf_mod, stack, M, nf, push)
    src = torch.from_numpy(stack.view(np.int16)).pin_memory().numpy().view(np.uint16) if pinned else stack
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(80, 96, M, 1.5, 2, nf, nf, framesPerLaunch=4)
    outs = [torch.empty((4, 96 * M, 80 * M), dtype=torch.float32).pin_memory().numpy() for _ in range(5)]
    try:
        for b in range(5):
            eng.resetFramePosition()
            for s in range(0, nf, push):
                assert not eng.calculateSRRF(src[b * nf + s:b * nf + s + push])
            eng.readSRRFbufferAsync(outs[b])  # five queued reads over two slots
        eng.finishQueue()
        # a synchronous read after queued ones
        eng.resetFramePosition()
        assert not eng.calculateSRRF(src[:nf])
        again = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    for b in range(5):
        np.testing.assert_array_equal(outs[b], want[b])
    np.testing.assert_array_equal(again, want[0])


def test_async_reads_bicubic_mp_correction(esrrf_mod):
    """Queued read-backs on the bicubic path: the MP correction runs inside each queued read, so
    five blocks read through two slots equal synchronous reads bit for bit, and the MP maps read
    after the last queued block are that block's."""
    import torch
    from esrrf import synth
    stack = synth.small_stack(5, 30, 40, 56)  # 5 blocks of 6 frames
    M, nf = 4, 6

    def engine():
        e = esrrf_mod.LiveSRRF_CL()
        e.initialise(56, 40, M, 1.5, 2, nf, nf, doMPmapCorrection=True, doFHTinterpolation=False)
        return e

    want, maps = [], None
    eng = engine()
    try:
        for b in range(5):
            eng.resetFramePosition()
            assert not eng.calculateSRRF(stack[b * nf:(b + 1) * nf])
            want.append(eng.readSRRFbuffer().copy())
        maps = eng.readMPmaps()
    finally:
        eng.release()
    outs = [torch.empty((4, 40 * M, 56 * M), dtype=torch.float32).pin_memory().numpy() for _ in range(5)]
    eng = engine()
    try:
        for b in range(5):
            eng.resetFramePosition()
            assert not eng.calculateSRRF(stack[b * nf:(b + 1) * nf])
            eng.readSRRFbufferAsync(outs[b])
        eng.finishQueue()
        got_maps = eng.readMPmaps()
    finally:
        eng.release()
    for b in range(5):
        np.testing.assert_array_equal(outs[b], want[b])
    np.testing.assert_array_equal(got_maps, maps)
