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
