"""The FP32 ABFT threshold of the mixed-precision form (ensemble.fp32_d1_threshold).

The threshold is a probabilistic rounding-error bound built from the
checksum weights w = A 1_int and w_abs = |A| 1_int.  These tests pin the
host computation of the weights to the oracle's w_A (the weights the
library's checksum uses) and check the bound's basic properties.
"""
import numpy as np
import pytest

from mnhack8_b200.ensemble import checksum_weights, fp32_d1_threshold
from oracle import oracle as orc


@pytest.mark.parametrize("N", [4, 7])
def test_weights_match_oracle(N):
    rng = np.random.default_rng(N)
    k = np.exp(rng.normal(0.0, 1.0, N ** 3))
    r = rng.uniform(0.5, 2.0, N ** 3)
    dt = 1e-3
    w, wabs = checksum_weights(N, k, r, dt)
    o = orc.Oracle(N, dt, k, r, detect=True)
    wA = o.vectors()["wA"].reshape((N + 1,) * 3)
    inner = np.zeros((N + 1,) * 3, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    np.testing.assert_allclose(w[inner], wA[inner], rtol=1e-12, atol=0)
    assert np.all(w[~inner] == 0.0)
    assert np.all(wabs >= np.abs(w) - 1e-15 * np.abs(wabs))


def test_pure_mass_has_no_cancellation():
    N = 5
    k, r = np.ones(N ** 3), np.ones(N ** 3)
    w, wabs = checksum_weights(N, k, r, 0.0)
    np.testing.assert_allclose(wabs, w, rtol=1e-14)
    # ||w_abs|| / ||w|| = 1: the bound is lam sqrt(depth) u / sqrt(n_int)
    thr = fp32_d1_threshold(N, k, r, 0.0)
    assert thr == pytest.approx(6.0 * 4.0 * 2.0 ** -24 / np.sqrt((N - 1) ** 3), rel=1e-12)


def test_threshold_grows_with_stiffness():
    N = 8
    rng = np.random.default_rng(1)
    k = np.exp(rng.normal(0.0, 1.5, N ** 3))
    r = np.ones(N ** 3)
    t_small = fp32_d1_threshold(N, k, r, 1e-6)
    t_large = fp32_d1_threshold(N, k, r, 1e-2)
    assert 0.0 < t_small < t_large < 1e-5
