"""GPU test of the device-side failure detection, without a GPU fault: the tensor-core passes'
bounded mbarrier wait, run on a barrier that nothing arrives at with a short limit (about a
millisecond of SM clock), gives up, records it in a device flag, and the host reads
ESRRF_ERR_TIMEOUT; the same wait with its arrival returns at once; the context stays usable (a
block computes normally afterwards).  The reference's waits are host-side queue.finish() calls
(LiveSRRF_CL.java:737-740, 1009-1015); this is the engine's own mechanism."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OK, TIMEOUT, INVALID = 0, -5, -1


def test_wait_without_arrival_times_out_and_the_context_stays_usable(esrrf_mod, oracle_mod):
    L = esrrf_mod.lib()
    assert L.esrrf_check_bounded_wait(0, 1, 2_000_000) == OK
    assert L.esrrf_check_bounded_wait(0, 0, 2_000_000) == TIMEOUT
    assert L.esrrf_check_bounded_wait(0, 0, 0) == INVALID
    assert L.esrrf_check_bounded_wait(0, 1, 2_000_000) == OK
    from esrrf import synth
    from conftest import rel_err
    raw = synth.small_stack(90, 6, 32, 32, emitters=8)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(32, 32, 2, 1.5, 1, 6, 6)
    try:
        eng.resetFramePosition()
        assert not eng.calculateSRRF(raw)
        got = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw.astype(np.float32), 2), 2, 1.5, 1)
    for k in range(4):
        assert rel_err(got[k], ref[k]) < 1e-4, k
