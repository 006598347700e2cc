"""The Philox restatement used to check the ensemble's on-device noise:
the published round structure gives distinct, uniform outputs and standard
normal deviates."""
import numpy as np

import philox_ref  # oracle/ is on sys.path (conftest)


def test_philox_outputs_distinct_and_uniform():
    u1, u2 = philox_ref.uniforms(20240611, 3, 1 << 16)
    both = np.concatenate([u1, u2])
    assert len(np.unique(both)) == len(both)
    hist, _ = np.histogram(both, bins=64, range=(0.0, 1.0))
    expected = len(both) / 64
    chi2 = float(((hist - expected) ** 2 / expected).sum())
    assert chi2 < 120.0  # 63 degrees of freedom


def test_philox_counter_and_key_change_the_stream():
    a = philox_ref.noise(7, 1, 1000, 1.0)
    assert not np.allclose(a, philox_ref.noise(8, 1, 1000, 1.0))
    assert not np.allclose(a, philox_ref.noise(7, 2, 1000, 1.0))
    assert np.array_equal(a, philox_ref.noise(7, 1, 1000, 1.0))
    # the first n points do not depend on n
    assert np.array_equal(a[:999], philox_ref.noise(7, 1, 999, 1.0))


def test_philox_normals():
    z = philox_ref.noise(123, 5, 400000, 1.0)
    assert abs(z.mean()) < 0.01
    assert abs(z.std() - 1.0) < 0.01
    assert abs((z ** 4).mean() - 3.0) < 0.05
