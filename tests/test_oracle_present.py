"""The present pass (captureFrame colorSpace 'output') of the CPU oracle against
the reference's tonemap known answers (shared-samplers/src/__tests__/tonemap.test.ts)."""
import numpy as np

import oracle


def test_aces_is_zero_at_zero_bounded_and_monotonic():
    x = np.array([0.0, 0.2, 0.5, 1.0, 10.0, 1e6])
    y = oracle.present(x, 0, 1.0, srgb=False)
    assert abs(y[0]) < 1e-6 and y.max() <= 1.0 and np.all(np.diff(y) >= 0) and y[2] > y[1]


def test_reinhard_known_values():
    y = oracle.present(np.array([0.0, 1.0, 3.0, -0.5]), 2, 1.0, srgb=False)
    assert np.allclose(y, [0.0, 0.5, 0.75, 0.0])


def test_agx_bounded_and_increasing_in_the_mid_range():
    y = oracle.present(np.array([0.0, 0.05, 1.0, 1e6]), 1, 1.0, srgb=False)
    assert y[0] >= 0 and y[3] <= 1 and y[2] > y[1]


def test_exposure_linear_none_and_srgb():
    assert np.allclose(oracle.present(np.array([0.25, 4.0]), 4, 2.0, srgb=False), [0.5, 8.0])
    assert np.allclose(oracle.present(np.array([0.25, 4.0]), 3, 2.0, srgb=False), [0.5, 1.0])
    assert np.allclose(oracle.present(np.array([0.0, 1.0, 0.001]), 3, 1.0, srgb=True), [0.0, 1.0, 0.01292])
    assert np.allclose(oracle.present(np.array([np.nan, 1.0]), 4, 0.0, srgb=False), [0.0, 0.0])
