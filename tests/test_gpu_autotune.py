"""GPU tests of the engine's autotuner (esrrf_create with frames_per_launch =
ESRRF_FRAMES_PER_LAUNCH_TUNED): it measures the candidates on first use, caches the choice per
parameter set and reuses it, the choice is within 2 % of the best candidate re-measured here, and
the tuned engine computes the same block as one with that launch size given explicitly.

The reference's counterpart sizes its GPU loads from a memory model (calculatenFrameOnGPU /
predictMemoryUsed, gui/LiveSRRF_optimised_.java:763-877)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def block_ms(esrrf, raw, M, F, reps=3, **kw):
    import torch

    eng = esrrf.LiveSRRF_CL()
    n = raw.shape[0]
    eng.initialise(raw.shape[-1], raw.shape[-2], M, 1.5, 2, n, n, framesPerLaunch=F, **kw)
    try:
        import ctypes

        d = torch.from_numpy(raw.astype(np.float32)).cuda()
        L = esrrf.lib()
        H = eng.handle
        out = torch.empty((4, raw.shape[-2] * M, raw.shape[-1] * M), dtype=torch.float32, device="cuda")
        best = 1e30
        for r in range(reps + 1):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
            esrrf._lib.check(H, L.esrrf_calculate_srrf_f32_device(H, ctypes.c_void_p(d.data_ptr()), n))
            esrrf._lib.check(H, L.esrrf_read_srrf_device(H, ctypes.c_void_p(out.data_ptr())))
            e1.record()
            torch.cuda.synchronize()
            if r:
                best = min(best, e0.elapsed_time(e1))
        return best, out.cpu().numpy(), eng.framesPerLaunch(), eng.tuneReport()
    finally:
        eng.release()


def test_tuned_launch_size_is_cached_and_near_the_best(esrrf_mod, tmp_path, monkeypatch):
    from esrrf import synth

    monkeypatch.setenv("ESRRF_TUNE_CACHE", str(tmp_path / "tune.txt"))
    raw = synth.small_stack(81, 60, 256, 256, emitters=60)
    M = 4
    _, out_a, F_a, rep_a = block_ms(esrrf_mod, raw, M, "auto", reps=0)
    assert rep_a["source"] == "measured" and rep_a["frames_per_launch"] == F_a
    cands = {c["frames_per_launch"] for c in rep_a["candidates"]}
    assert F_a in cands and len(cands) >= 3
    # a second engine with the same parameters reads the cache, measures nothing
    _, out_b, F_b, rep_b = block_ms(esrrf_mod, raw, M, "auto", reps=0)
    assert rep_b["source"] == "cache" and F_b == F_a
    np.testing.assert_array_equal(out_a, out_b)
    assert (tmp_path / "tune.txt").read_text().count("\n") == 1
    # re-measure every candidate with an explicit launch size: the tuned one within 2 % of the best
    times = {F: block_ms(esrrf_mod, raw, M, F)[0] for F in sorted(cands)}
    best = min(times, key=times.get)
    if times[F_a] > 1.02 * times[best]:
        # a shared GPU's timing noise: re-time the two contenders, more repetitions each
        times[F_a] = block_ms(esrrf_mod, raw, M, F_a, reps=8)[0]
        times[best] = block_ms(esrrf_mod, raw, M, best, reps=8)[0]
    assert times[F_a] <= 1.02 * min(times.values()), (F_a, times)
    # and the explicit launch size computes the same block
    _, out_e, _, rep_e = block_ms(esrrf_mod, raw, M, F_a, reps=0)
    assert rep_e["source"] == "off"
    for k in range(4):
        assert rel_err(out_a[k], out_e[k]) < 1e-5


def test_tuner_picks_a_3d_kernel_form(esrrf_mod, tmp_path, monkeypatch):
    """In 3-D the candidates also cover the tabulated kernel's forms (two cells per thread, one
    cell per thread with the slab in shared memory, the field through L1); the tuned engine gives
    the oracle's block."""
    from esrrf import synth
    from oracle import oracle as O
    from test_gpu_bic3d import calib, run, tile_planes

    monkeypatch.setenv("ESRRF_TUNE_CACHE", str(tmp_path / "tune3d.txt"))
    P, n, hs, ws, M = 4, 6, 20, 24, 3
    planes = synth.small_stack(9, n, hs, ws, planes=P).astype(np.float32)
    theta = np.array([0.3, -0.5, 0.0, 0.8], np.float32)
    sx = np.array([0.1, -0.2, 0.0, 0.3], np.float32)
    sy = np.array([-0.1, 0.2, 0.0, 0.1], np.float32)
    roi = np.array([0, 1, 2, 3], np.float32)
    ref = O.block3d(planes, M, 1.5, 1, theta, sx, sy, mp_correction=True)
    got, _ = run(esrrf_mod, tile_planes(planes, roi), M, 1.5, 1, calib=calib(P, theta, sx, sy, roi),
                   frames_per_launch="auto")
    for k in range(4):
        assert rel_err(got.reshape(4, -1)[k], ref.reshape(4, -1)[k]) < 1e-4, k
    cache = (tmp_path / "tune3d.txt").read_text().split()
    assert len(cache) == 4 and cache[0].startswith("v1|") and "|3d|" in cache[0]
    assert int(cache[2]) in (1, 2, 3)  # a form was measured and chosen
