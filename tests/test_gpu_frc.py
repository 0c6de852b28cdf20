"""GPU tests of esrrf_frc (the sweep's FRC resolution, gui/ParametersSweep_.java:403-447) against
the float64 oracle (oracle/frc_oracle.py): curves within 2e-5 (FP32 FFT, FP64 ring sums), FIRE
within 1e-4 relative, NaN where the oracle has none; padded sizes 32 .. 2048, ragged images,
batches, pixel size; and the sweep's odd/even FRC mode end to end."""
import math

import numpy as np
import pytest

from conftest import rel_err
from oracle import frc_oracle as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("h,w", [(80, 100), (19, 37), (512, 512), (700, 1000), (1500, 2048)])
def test_frc_matches_oracle(esrrf_mod, h, w):
    pairs = [F.split_images(10 + i, h, w, c, s) for i, (c, s) in enumerate([(0.05, 5.0), (0.15, 10.0), (0.3, 2.0)])]
    A = np.stack([p[0] for p in pairs]).astype(np.float32)
    B = np.stack([p[1] for p in pairs]).astype(np.float32)
    fire, curves = esrrf_mod.frc(A, B, curves=True)
    N, R = esrrf_mod.frc_size(w, h)
    assert N == F.padded_size(w, h) and curves.shape == (3, R)
    for i in range(3):
        want, c = F.fire(A[i], B[i])
        assert np.abs(curves[i] - c).max() < 2e-5, (i, np.abs(curves[i] - c).max())
        if math.isnan(want):
            assert math.isnan(fire[i])
        else:
            assert abs(fire[i] - want) <= 1e-4 * want, (i, fire[i], want)


def test_frc_nan_cases_and_pixel_size(esrrf_mod):
    a, b = F.split_images(3, 64, 64, 0.1, 5.0)
    same = esrrf_mod.frc(np.stack([a, a]).astype(np.float32), np.stack([a, a]).astype(np.float32))
    assert np.isnan(same).all()
    r1 = esrrf_mod.frc(a.astype(np.float32), b.astype(np.float32))[0]
    r2 = esrrf_mod.frc(a.astype(np.float32), b.astype(np.float32), pixel_size=0.0265)[0]
    assert r2 == pytest.approx(r1 * 0.0265, rel=1e-6)
    with pytest.raises(esrrf_mod.EsrrfError):
        esrrf_mod.frc_size(5000, 10)


def test_sweep_frc_mode(esrrf_mod, oracle_mod):
    """Odd frames (0, 2, 4, ... 0-based) and even frames reconstructed separately, FIRE of each
    cumulant pair in raw-pixel-size / M units."""
    from esrrf import synth
    stack = synth.small_stack(21, 20, 40, 48)
    res, odd, even = esrrf_mod.sweep_frc(stack, [2], [1.0, 1.5], [1, 2], 10, pixel_size=0.1)
    assert set(res) == {(2, 1.0, 1), (2, 1.0, 2), (2, 1.5, 1), (2, 1.5, 2)}
    for M, r, S in res:
        for half, start in ((odd, 0), (even, 1)):
            raw = stack[start:20:2].astype(np.float32)
            ref = oracle_mod.fht_block(oracle_mod.fht_interpolate(raw, M), M, r, S)
            for k in range(4):
                assert rel_err(half[(M, r, S)][k], ref[k]) < 1e-4, (M, r, S, start, k)
        for c, name in enumerate(("AVG", "VAR", "TAC2")):
            want = F.fire(odd[(M, r, S)][c], even[(M, r, S)][c], pixel_size=0.1 / M)[0]
            got = res[(M, r, S)][name]
            assert (math.isnan(want) and math.isnan(got)) or abs(got - want) <= 1e-3 * want, (M, r, S, name, got, want)
