"""TEST INFRASTRUCTURE -- not part of the product.

numpy restatement of FIRTEZ-dz's line spread function, the checker of the
library's LSF kernels (fz_lsf_gaussian / fz_lsf_kernel and the convolution
pass of the synthesis and response-function launches).

Followed (src/ unless noted):
  LSF_INIT pre_post_duties.f90:742-900 -- the Gaussian kernel of each
      spectral region (positions 1..SKI centred, in mA of WAVE(WI+1) -
      WAVE(WI), half a step off for even SKI, exp(-(x - W0 - WOFF)^2 /
      (2 SIGMA^2)), normalised, CSHIFT by SKI/2), the validity test
      |sum - 1| < 0.01 and the second normalisation; LSF_KERNEL = YK / SKI
      transformed once (FFTW r2c)
  CALCULATE_EQUIVALENT_SYN1D forward.f90:793-853 and the MLSF branches of
      CALCULATE_EQUIVALENT_DSYN :615-657, :736-772 -- per region r2c of
      DBLE(row), times the kernel's transform, c2r (FFTW's unnormalised
      inverse), REAL(.)
numpy's pocketfft stands in for FFTW 3.3.8 (the reference's version); the
two agree to ~1e-16 relative before the REAL*4 rounding.
"""
import numpy as np


def gaussian(n, wave_ini, dlambda, sigma, w0):
    """LSF_INIT's Gaussian YK (n values, centre at index 0), before the
    validity test."""
    dw = (wave_ini + dlambda * 1.0) - (wave_ini + dlambda * 0.0)
    xk = np.arange(1, n + 1, dtype=np.float64)
    xk = (xk - np.sum(xk) / float(n)) * dw
    woff = (xk[1] - xk[0]) / 2.0 if n % 2 == 0 else 0.0
    yk = np.exp(-((xk - w0 - woff) ** 2 / (2.0 * sigma ** 2)))
    yk = yk / np.sum(yk)
    return np.roll(yk, -(n // 2))   # CSHIFT(YK, SHIFT=n/2): result(i) = YK(i + n/2)


def install(yk):
    """(valid, kernel): |sum - 1| < 0.01, then YK / sum(YK)."""
    s = float(np.sum(yk))
    return abs(s - 1.0) < 0.01, np.asarray(yk, dtype=np.float64) / s


def convolve(rows, numwave, kernels, valid):
    """rows (..., NUMW) (any float type; DBLE taken) -> REAL*4 rows, each
    region convolved with its kernel (kernels: one array per region)."""
    out = np.array(rows, dtype=np.float64, copy=True)
    o = 0
    for n, k, v in zip(numwave, kernels, valid):
        if v:
            seg = out[..., o:o + n]
            ft = np.fft.rfft(seg, axis=-1) * np.fft.rfft(np.asarray(k) / float(n))
            out[..., o:o + n] = np.fft.irfft(ft, n=n, axis=-1) * float(n)
        o += n
    return out.astype(np.float32)
