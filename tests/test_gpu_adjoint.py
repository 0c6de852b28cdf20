"""GPU tests of the differentiable eSRRF adjoint (esrrf_loss_and_grad): the loss against the FP64
reference loss, and every gradient (radius, sensitivity, re-blur sigma, input pixels) against
central finite differences (h = 1e-3) of the FP64 reference, to 1e-3 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    from esrrf import synth
    raw = synth.small_stack(71, 6, 24, 24, emitters=10).astype(np.float32)
    return raw, 3, 1.5, 2.0, 1.3  # frames, M, radius, sensitivity, re-blur sigma


def test_loss_matches_fp64(esrrf_mod, case):
    from oracle import adjoint_oracle as A
    raw, M, fwhm, S, sig = case
    adj = esrrf_mod.Adjoint(24, 24, 6, M)
    try:
        L = adj.loss(raw, fwhm, S, sig)
    finally:
        adj.release()
    L64 = A.loss(raw, M, fwhm, S, sig)
    assert abs(L - L64) <= 1e-4 * abs(L64), (L, L64)


def test_gradients_match_finite_differences(esrrf_mod, case):
    from oracle import adjoint_oracle as A
    raw, M, fwhm, S, sig = case
    rng = np.random.default_rng(0)
    pix = [(int(rng.integers(6)), int(rng.integers(24)), int(rng.integers(24))) for _ in range(8)]
    pix += [(0, 0, 0), (5, 23, 23), (2, 0, 17)]  # borders
    fd = A.fd_gradient(raw, M, fwhm, S, sig, pixels=pix)
    adj = esrrf_mod.Adjoint(24, 24, 6, M)
    try:
        L, g, gf = adj.loss_and_grad(raw, fwhm, S, sig)
        gf = gf.cpu().numpy()
        # a second call on the same handle gives the same result
        L2, g2, gf2 = adj.loss_and_grad(raw, fwhm, S, sig)
    finally:
        adj.release()
    for k in ("fwhm", "S", "sigma"):
        assert abs(g[k] - fd[k]) <= 1e-3 * abs(fd[k]), (k, g[k], fd[k])
        assert abs(g2[k] - g[k]) <= 1e-6 * abs(g[k])
    scale = max(abs(v) for v in fd["pixels"].values())
    for (t, y, x), v in fd["pixels"].items():
        assert abs(gf[t, y, x] - v) <= 1e-3 * max(abs(v), 0.05 * scale), ((t, y, x), gf[t, y, x], v)
    np.testing.assert_allclose(gf2.cpu().numpy(), gf, rtol=1e-4, atol=1e-6 * scale)


def test_gradient_search_descends(esrrf_mod, case):
    raw, M, fwhm, S, sig = case
    adj = esrrf_mod.Adjoint(24, 24, 6, M)
    try:
        traj = esrrf_mod.gradient_search(adj, raw, 1.2, 1.5, 1.0, steps=6)
    finally:
        adj.release()
    losses = [l for _, l in traj]
    assert len(losses) >= 2 and all(b < a for a, b in zip(losses, losses[1:]))
