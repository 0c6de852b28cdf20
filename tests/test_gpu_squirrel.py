"""GPU tests of esrrf_squirrel (SQUIRREL metrics of ErrorMapLiveSRRF.java as the parameter sweep
applies them) against the float64 restatement in oracle/squirrel_oracle.py: a known answer, every
reconstruction of a small sweep (AVG, VAR, TAC2 scored against the block's INT slice), and the
crop, fixed-sigma and error-map options.

Tolerances: the GPU blurs in FP32 and sums in FP64, so the objective differs from the oracle's at
~1e-7 relative and the minimising sigma, where the RMSE is flat, moves by up to ~1e-3 relative;
alpha and beta follow sigma to first order, RSE and RSP to second order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def close(got, ref, what):
    assert abs(got["sigma"] - ref["sigma"]) <= 2e-3 * max(ref["sigma"], 0.1), (what, "sigma", got["sigma"], ref["sigma"])
    assert abs(got["alpha"] - ref["alpha"]) <= 5e-3 * abs(ref["alpha"]) + 1e-6, (what, "alpha", got["alpha"], ref["alpha"])
    assert abs(got["rse"] - ref["rse"]) <= 1e-4 * ref["rse"] + 1e-6, (what, "rse", got["rse"], ref["rse"])
    assert abs(got["rsp"] - ref["rsp"]) <= 1e-5, (what, "rsp", got["rsp"], ref["rsp"])


def test_known_answer(esrrf_mod):
    from oracle import squirrel_oracle as Q
    rng = np.random.default_rng(7)
    x = Q.blur(rng.random((96, 80)) * 100.0, 1.0).astype(np.float32)
    ref = (2.5 * Q.blur(x, 1.7) + 10.0).astype(np.float32)
    m = esrrf_mod.squirrel(x[None], ref, 2)
    assert abs(m["sigma"][0] - 1.7) < 2e-3 and abs(m["alpha"][0] - 2.5) < 1e-3 and abs(m["beta"][0] - 10.0) < 0.05
    assert m["rsp"][0] > 1 - 1e-6


def test_sweep_reconstructions_match_oracle(esrrf_mod):
    from esrrf import synth
    from oracle import squirrel_oracle as Q
    raw = synth.small_stack(3, 30, 48, 40)
    sw = esrrf_mod.Sweep(40, 48, 30, [2, 3], [1.0, 1.5], [1, 2], [(0, 30), (5, 17)])
    try:
        res = sw.run(raw)
        got = sw.squirrel(res)
    finally:
        sw.release()
    assert len(got) == 2 * 2 * 2 * 2
    for k, v in res.items():
        for c, name in enumerate(("AVG", "VAR", "TAC2")):
            close(got[k][name], Q.squirrel(v[c], v[3], k[0]), f"{k} {name}")


def test_crop_fixed_sigma_and_error_maps(esrrf_mod):
    from esrrf import synth
    from oracle import squirrel_oracle as Q
    raw = synth.small_stack(9, 20, 40, 40)
    res = esrrf_mod.rolling(raw, 3, 1.5, 1, [(0, 20)])[(0, 20)]
    sr = np.stack([res[0], res[1]])
    for kw in (dict(crop=2), dict(fixed_sigma=0.6), dict(crop=1, fixed_sigma=0.9)):
        m = esrrf_mod.squirrel(sr, res[3], 3, error_maps=True, **kw)
        for i in range(2):
            ref = Q.squirrel(sr[i], res[3], 3, **kw)
            close({f: m[f][i] for f in ("sigma", "alpha", "rse", "rsp")}, ref, str(kw))
            e = ref["error_map"]
            assert m["error_map"][i].shape == e.shape
            assert np.abs(m["error_map"][i] - e).max() <= 2e-3 * (e.max() - e.min()) + 1e-4, kw
