"""CPU checks of the float64 SQUIRREL restatement (oracle/squirrel_oracle.py) that the GPU
metrics are tested against: the Brent search against scipy's bounded Brent, the blur's edge
handling, and a known answer (a reference made by blurring, scaling and offsetting the image)."""
import numpy as np
import pytest


def test_brent_matches_scipy_bounded():
    from scipy.optimize import minimize_scalar
    from oracle import squirrel_oracle as Q
    for f in (lambda x: (x - 0.3) ** 2 + 0.1 * np.sin(3 * x), lambda x: np.cosh(x - 2.2), lambda x: abs(x - 1.1) ** 1.5):
        x = Q.brent(f, 0.0, 3.4)
        ref = minimize_scalar(f, bounds=(0.0, 3.4), method="bounded", options={"xatol": 1e-12}).x
        assert abs(x - ref) < 1e-5, (x, ref)


def test_blur_keeps_constants_and_mass():
    from oracle import squirrel_oracle as Q
    c = np.full((37, 23), 3.25)
    np.testing.assert_allclose(Q.blur(c, 2.7), c, rtol=1e-12)
    rng = np.random.default_rng(1)
    x = rng.random((64, 64))
    np.testing.assert_array_equal(Q.blur(x, 0.0), x)  # sigma 0: no blur
    y = np.zeros((41, 41))
    y[20, 20] = 1.0
    assert abs(Q.blur(y, 1.5).sum() - 1.0) < 1e-12  # away from the edges the kernel sums to one


@pytest.mark.parametrize("sigma0,M", [(1.7, 2), (0.8, 3)])
def test_known_answer(sigma0, M):
    from oracle import squirrel_oracle as Q
    rng = np.random.default_rng(7)
    x = Q.blur(rng.random((96, 80)) * 100.0, 1.0)
    ref = 2.5 * Q.blur(x, sigma0) + 10.0
    m = Q.squirrel(x, ref, M)
    assert abs(m["sigma"] - sigma0) < 1e-4 and abs(m["alpha"] - 2.5) < 1e-6 and abs(m["beta"] - 10.0) < 1e-4
    assert m["rse"] < 1e-9 and m["rsp"] > 1 - 1e-12
