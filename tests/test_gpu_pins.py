"""The GPU's Voigt function and formal solution against independent
mathematics (the same pins as tests/test_pins_analytic.py for the oracle):

* fz_voigt (the FP32 Voigt of the synthesis kernels) against
  scipy.special.wofz: the HAW approximation's 5e-6 plus FP32 rounding,
  6e-6 absolute, for damping 1e-4 .. 3 and |v| <= 25;
* fz_rte_solve (the synthesis kernels' FP32 evolution operator and
  recursion) against the same recursion on scipy.linalg.expm operators,
  within 2e-6 of the largest Stokes value (FP32 over 24 layers), and
  against the Unno-Rachkovsky solution of a Milne-Eddington slab of 4000
  layers within 3e-5 (the scheme's own 3.5e-6 plus FP32 accumulation).
"""
import numpy as np
import pytest
from scipy.special import wofz

import test_pins_analytic as pins

pytestmark = pytest.mark.gpu


def test_gpu_voigt_is_the_faddeeva_function(fz):
    v = np.linspace(-25.0, 25.0, 4001, dtype=np.float32)
    for a in (1e-4, 1e-3, 1e-2, 0.1, 0.5, 1.0, 3.0):
        h, f = fz.voigt(np.float32(a), v)
        w = wofz(v.astype(np.float64) + 1j * np.float64(np.float32(a)))
        assert np.max(np.abs(h - w.real)) < 6e-6, a
        assert np.max(np.abs(f - w.imag)) < 6e-6, a


def test_gpu_formal_solution_is_the_matrix_exponential_recursion(fz, orc):
    rng = np.random.default_rng(7)
    ncol, nz, nw = 3, 24, 5
    eta = np.stack([np.stack([pins.zeeman_like_eta(rng, nw, 1e-7) for _ in range(nz)]) for _ in range(ncol)])
    eta = eta.astype(np.float32)
    zz = np.cumsum(rng.uniform(5.0, 40.0, nz))
    src = rng.uniform(0.5, 2.0, (ncol, nz, nw)).astype(np.float32)
    bnd = np.zeros((ncol, nz), dtype=np.int32)
    bnd[1, 6] = 1
    got = fz.rte_solve(eta, src, zz, bnd)
    for c in range(ncol):
        b = bnd[c] if bnd[c].any() else None
        ref = pins.expm_solution(eta[c].astype(np.float64), src[c].astype(np.float64), zz, b)
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(got[c] - ref)) < 2e-6 * scale, c
        assert np.max(np.abs(got[c] - orc.rte_solve(eta[c], src[c], zz, b))) < 2e-6 * scale, c


def test_gpu_unno_rachkovsky(fz):
    s0, s1 = 0.4, 1.3
    eta, tau, zz, kt = pins.me_slab(4001, 40.0, np.random.default_rng(3))
    tnext = np.concatenate([tau[1:], [0.0]])
    src = np.repeat((s0 + s1 * 0.5 * (tau + tnext))[:, None], eta.shape[2], axis=1)
    got = fz.rte_solve(eta[None].astype(np.float32), src[None].astype(np.float32), zz)[0]
    for lam in range(kt.shape[1]):
        ur = s0 * np.eye(4)[0] + s1 * np.linalg.solve(pins.absorption_matrix(*kt[:, lam]), np.eye(4)[0])
        assert np.max(np.abs(got[lam] - ur)) < 3e-5, (lam, got[lam], ur)
