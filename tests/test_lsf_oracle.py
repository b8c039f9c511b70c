"""The LSF oracle's restatement of LSF_INIT and the FFT convolution
(oracle/lsf_oracle.py) against properties that pin it: the Gaussian kernel
sums to 1 with its centre at index 0 (odd and even sizes, the even size's
half-step offset), a shifted centre w0 moves the peak by w0 / step, a delta
kernel is the identity, a constant row stays constant, and the circular
convolution equals the direct sum."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import lsf_oracle as lo  # noqa: E402


def test_gaussian_kernel_shape():
    for n in (7, 8, 112):
        k = lo.gaussian(n, -1193.25, 21.5, 30.0, 0.0)
        assert abs(k.sum() - 1.0) < 1e-14
        assert np.argmax(k) == 0
        # symmetric about index 0: k[j] == k[-j]
        np.testing.assert_allclose(k[1:n // 2], k[::-1][:n // 2 - 1], rtol=1e-12)
    k = lo.gaussian(112, -1193.25, 21.5, 30.0, 3 * 21.5)
    assert np.argmax(k) == 3


def test_convolution_identities():
    rng = np.random.default_rng(1)
    rows = rng.standard_normal((5, 30))
    delta = np.zeros(13)
    delta[0] = 1.0
    g = lo.gaussian(17, 0.0, 10.0, 12.0, 0.0)
    out = lo.convolve(rows, [13, 17], [delta, g], [True, True])
    np.testing.assert_array_equal(out[:, :13], rows[:, :13].astype(np.float32))
    direct = np.zeros((5, 17))
    for i in range(17):
        for j in range(17):
            direct[:, i] += rows[:, 13 + j] * g[(i - j) % 17]
    np.testing.assert_allclose(out[:, 13:], direct.astype(np.float32), rtol=2.4e-7, atol=1e-12)
    const = lo.convolve(np.full((1, 30), 0.75), [13, 17], [delta, g], [True, True])
    np.testing.assert_allclose(const, 0.75, rtol=1e-7)
    # an invalid region is left as it is
    out = lo.convolve(rows, [13, 17], [delta, g], [True, False])
    np.testing.assert_array_equal(out[:, 13:], rows[:, 13:].astype(np.float32))
    assert lo.install(g * 0.5)[0] is False and lo.install(g)[0] is True
