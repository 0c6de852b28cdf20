"""GPU parity tests of the 2-D FHT path (liveSRRF_noInterpolation.cl semantics) through the C ABI.

Tolerance: every output slice (AVG, VAR, TAC2, INT) must agree with the oracle within 1e-4 of
that slice's dynamic range (max - min), the bar the engine is specified to.  The oracle is the
FP32 restatement, itself pinned bit-exactly to the reference kernels by tests/test_oracle.py.
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-4


def run_engine(esrrf, frames, M, fwhm, S, intw=True, kernel="fused", drift=None,
               frames_per_launch=0, block=None, chunks=None):
    eng = esrrf.LiveSRRF_CL()
    n = frames.shape[0] if block is None else block
    eng.initialise(frames.shape[-1], frames.shape[-2], M, fwhm, S, n, n, intWeighting=intw,
                   kernel=kernel, framesPerLaunch=frames_per_launch)
    try:
        eng.resetFramePosition()
        if drift is not None:
            eng.loadDriftXYGPUbuffer(*drift)
        if chunks is None:
            assert not eng.calculateSRRF(frames)
        else:
            s = 0
            for c in chunks:
                assert not eng.calculateSRRF(frames[s:s + c])
                s += c
        return eng.readSRRFbuffer().copy()
    finally:
        eng.release()


def assert_close(got, ref, tol=TOL, what=""):
    for k in range(4):
        e = rel_err(got[k], ref[k])
        assert e < tol, f"{what} slice {k}: {e:.3g} of range"


@pytest.mark.parametrize("kernel", ["fused", "plain"])
@pytest.mark.parametrize("name", golden_names("fht"))
def test_fht_golden(esrrf_mod, name, kernel):
    g = load_golden(name)
    drift = (g["drift_x"], g["drift_y"]) if "drift_x" in g else None
    got = run_engine(esrrf_mod, g["raw"], int(g["magnification"]), float(g["fwhm"]),
                     int(g["sensitivity"]), bool(g["int_weighting"]), kernel=kernel, drift=drift)
    assert_close(got, g["out"], what=f"{name}/{kernel}")


def test_fht_u16_input_and_chunked_pushes(esrrf_mod, oracle_mod):
    """uint16 frames pushed in uneven GPU loads give the same block as one float push."""
    from esrrf import synth
    raw = synth.small_stack(21, 13, 32, 32)
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw.astype(np.float32), 4), 4, 1.5, 2)
    got = run_engine(esrrf_mod, raw, 4, 1.5, 2, chunks=[5, 1, 7], frames_per_launch=3)
    assert_close(got, ref, what="u16 chunked")
    got2 = run_engine(esrrf_mod, raw.astype(np.float32), 4, 1.5, 2)
    assert_close(got2, ref, what="f32 single push")


def test_fht_workload_fht64_subset(esrrf_mod, oracle_mod):
    """The 64x64, M5, radius 1.5, S1 workload on its first 20 frames, fused and plain."""
    from esrrf import synth
    raw = synth.make_stack("fht64", frames=20)
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw.astype(np.float32), 5), 5, 1.5, 1)
    for kernel in ("fused", "plain"):
        got = run_engine(esrrf_mod, raw, 5, 1.5, 1, kernel=kernel)
        assert_close(got, ref, what=f"fht64/{kernel}")


def test_fht_mirror_padded_non_square(esrrf_mod, oracle_mod):
    from esrrf import synth
    raw = synth.small_stack(22, 6, 20, 28).astype(np.float32)
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw, 3), 3, 2.0, 1)
    got = run_engine(esrrf_mod, raw, 3, 2.0, 1)
    assert_close(got, ref, what="non-square")


@pytest.mark.parametrize("fwhm,M", [(0.5, 2), (1.0, 4), (2.5, 2), (3.0, 4)])
def test_fht_radius_range(esrrf_mod, oracle_mod, fwhm, M):
    """Radii of the parameter sweep (tap boxes from 6 to 26 wide) on both kernels."""
    from esrrf import synth
    raw = synth.small_stack(23, 5, 24, 24).astype(np.float32)
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw, M), M, fwhm, 2)
    for kernel in ("fused", "plain"):
        got = run_engine(esrrf_mod, raw, M, fwhm, 2, kernel=kernel)
        assert_close(got, ref, what=f"r{fwhm} M{M} {kernel}")


def test_intensity_scaling_property_full_size(esrrf_mod):
    """Size-independent property at the 512x512, M4 workload size: CGLH does not depend on the
    intensity scale, so scaling the frames by c scales AVG, INT by c and VAR, TAC2 by c^2."""
    from esrrf import synth
    raw = synth.make_stack("fht512", frames=12).astype(np.float32)
    a = run_engine(esrrf_mod, raw, 4, 1.5, 2)
    b = run_engine(esrrf_mod, raw * 2.0, 4, 1.5, 2)
    for k, p in zip(range(4), (1, 2, 2, 1)):
        assert rel_err(b[k], a[k] * 2.0 ** p) < TOL, k


def test_identical_frames_full_size(esrrf_mod):
    """Size-independent property at 512x512, M4: a block of identical frames has VAR = TAC2 = 0
    (up to rounding, relative to AVG^2) and INT equals the interpolated frame's values; the
    interpolation of a constant frame is the constant."""
    from esrrf import synth
    f = synth.make_stack("fht512", frames=1)
    out = run_engine(esrrf_mod, np.repeat(f, 6, axis=0), 4, 1.5, 2)
    scale = float((out[0].astype(np.float64) ** 2).max())
    assert np.abs(out[1]).max() <= 1e-5 * scale
    assert np.abs(out[2]).max() <= 1e-5 * scale
    c = np.full((3, 512, 512), 300, np.uint16)
    out = run_engine(esrrf_mod, c, 4, 1.5, 2)
    np.testing.assert_allclose(out[3], 300.0, rtol=1e-5)


def test_launch_split_and_time_reversal_full_size(esrrf_mod):
    """Size-independent properties of one 100-frame block at 512x512, M4 (the full block of the
    500-frame workload): the cumulants do not depend on how the block is cut into launches (the
    default 34 + 33 + 33, 8 per launch, uneven pushes of 17 + 50 + 33), and they are unchanged when
    the frames are taken in reverse order -- AVG, VAR and INT are sums over frames and TAC2 sums the
    products of adjacent frames, so a frame pair lost or counted twice at a launch edge shows."""
    from esrrf import synth
    raw = synth.make_stack("fht512", frames=100)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(512, 512, 4, 1.5, 2, 100, 100)
    try:
        assert eng.framesPerLaunch() == 34
    finally:
        eng.release()
    a = run_engine(esrrf_mod, raw, 4, 1.5, 2)
    b = run_engine(esrrf_mod, raw, 4, 1.5, 2, frames_per_launch=8)
    c = run_engine(esrrf_mod, raw, 4, 1.5, 2, chunks=[17, 50, 33])
    r = run_engine(esrrf_mod, np.ascontiguousarray(raw[::-1]), 4, 1.5, 2)
    assert_close(b, a, tol=1e-5, what="8 per launch")
    assert_close(c, a, tol=1e-5, what="uneven pushes")
    assert_close(r, a, tol=1e-5, what="reversed")
    assert np.abs(a[2]).max() > 0  # TAC2 carries signal in this block


def test_block_overflow_and_cancel(esrrf_mod):
    from esrrf import EsrrfError, synth
    raw = synth.small_stack(24, 6, 16, 16)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(16, 16, 2, 1.5, 1, 4, 4)
    try:
        eng.resetFramePosition()
        with pytest.raises(EsrrfError):
            eng.calculateSRRF(raw)  # 6 frames into a 4-frame block
        eng.resetFramePosition()
        eng.requestCancel()
        assert eng.calculateSRRF(raw[:4]) is True
    finally:
        eng.release()


def test_small_frames_split_into_frame_groups(esrrf_mod, oracle_mod):
    """Small frames (a 96 x 80 output is 6 CTA tiles) split each launch's frames into groups
    across CTAs: 20-frame launches in 5 groups, each later group re-running the frame before it
    for TAC2's previous value, sums folded atomically, the last values handed to the next launch.
    Same block as the oracle and as 3-frame launches (one group)."""
    from esrrf import synth
    raw = synth.small_stack(91, 40, 40, 48).astype(np.float32)
    ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw, 2), 2, 1.5, 2)
    grouped = run_engine(esrrf_mod, raw, 2, 1.5, 2, frames_per_launch=20, chunks=[20, 20])
    single = run_engine(esrrf_mod, raw, 2, 1.5, 2, frames_per_launch=3)
    assert_close(grouped, ref, what="grouped vs oracle")
    assert_close(grouped, single, tol=1e-5, what="grouped vs one group")
    assert np.abs(grouped[2]).max() > 0


def test_frames_of_the_wrong_size_are_rejected(esrrf_mod):
    """calculateSRRF checks the stack's frame size against initialise's (the library reads
    n x height x width values from the pointer it is given); a single 2-D frame is one frame."""
    from esrrf import EsrrfError, synth
    raw = synth.small_stack(26, 4, 24, 32)
    eng = esrrf_mod.LiveSRRF_CL()
    eng.initialise(32, 24, 2, 1.5, 1, 4, 4)
    try:
        eng.resetFramePosition()
        with pytest.raises(EsrrfError, match="frames must be"):
            eng.calculateSRRF(raw[:, :, :16])
        with pytest.raises(EsrrfError, match="frames must be"):
            eng.calculateSRRF(raw.transpose(0, 2, 1))
        for t in range(4):
            assert not eng.calculateSRRF(raw[t])
        one = eng.readSRRFbuffer().copy()
    finally:
        eng.release()
    ref = run_engine(esrrf_mod, raw, 2, 1.5, 1)  # the same block in one push
    for k in range(4):
        assert rel_err(one[k], ref[k]) < 1e-6, k
