"""The line spread function on the GPU against the oracle's restatement of
the reference's FFT convolution (oracle/lsf_oracle.py): the library's
convolution of the synthesis, of the node Jacobian and of the full-height
response functions equals the oracle's convolution of the same unconvolved
GPU output (REAL*4 results; the FP64 direct sum and the FFT differ by
~1e-16 before rounding: 1 ulp of REAL*4 at most, rtol 2.4e-7, atol 1e-15);
an invalid kernel leaves its region alone; an inversion with the LSF fits
observations made with it (chi2 at the true model near the noise level
with the LSF, far above it without)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import lmcase  # noqa: E402
import lsf_oracle as lo  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = dict(rtol=2.4e-7, atol=1e-15)


def _setup(fz, orc, nz):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    return fz.Synthesis(lines, reg, nz=nz, gain=g), reg


def _kernels(reg, params):
    ks, valid = [], []
    for r, (sigma, w0) in enumerate(params):
        k = lo.gaussian(int(reg["numwave"][r]), float(reg["wave_ini"][r]), float(reg["dlambda"][r]), sigma, w0)
        v, k = lo.install(k)
        ks.append(k)
        valid.append(v)
    return ks, valid


def test_synthesis_and_node_jacobian_with_lsf(fz, orc):
    ctx, reg = _setup(fz, orc, 48)
    nw = [int(n) for n in reg["numwave"]]
    m = fz.atmos.make_columns(12, 48, seed=4)
    ctx.rf_nodes(lmcase.NODES)
    syn0, _, st = ctx.forward(m, hydrostatic=True)
    rsyn0, jac0, _, _ = ctx.forward_rf(m, hydrostatic=True)
    params = [(30.0, 0.0), (45.0, 10.75)]
    for r, (sg, w0) in enumerate(params):
        assert ctx.lsf_gaussian(r, sg, w0)
    ks, valid = _kernels(reg, params)
    syn1, _, st1 = ctx.forward(m, hydrostatic=True)
    assert np.all(st == 0) and np.all(st1 == 0)
    np.testing.assert_allclose(syn1, lo.convolve(syn0, nw, ks, valid), **TOL)
    rsyn1, jac1, _, _ = ctx.forward_rf(m, hydrostatic=True)
    np.testing.assert_allclose(rsyn1, lo.convolve(rsyn0, nw, ks, valid), **TOL)
    j0 = jac0.reshape(jac0.shape[0], jac0.shape[1], 4, -1)
    np.testing.assert_allclose(jac1.reshape(j0.shape), lo.convolve(j0, nw, ks, valid), **TOL)
    # an invalid kernel (sum 0.5) leaves region 1 unconvolved
    k = np.zeros(nw[1])
    k[0] = 0.5
    assert not ctx.lsf_kernel(1, k)
    syn2, _, _ = ctx.forward(m, hydrostatic=True)
    np.testing.assert_allclose(syn2, lo.convolve(syn0, nw, ks, [True, False]), **TOL)
    ctx.lsf_clear()
    syn3, _, _ = ctx.forward(m, hydrostatic=True)
    np.testing.assert_array_equal(syn3, syn0)


def test_full_height_rfs_with_lsf(fz, orc):
    import torch
    nz = 24
    ctx, reg = _setup(fz, orc, nz)
    nw = [int(n) for n in reg["numwave"]]
    ncol = 3
    m = torch.from_numpy(fz.atmos.make_columns(ncol, nz, seed=9)).cuda()
    nf = 4 * ctx.numw

    def run():
        rf = torch.empty((ncol, 6, nz, nf), dtype=torch.float32, device="cuda")
        so = torch.empty((ncol, 4, ctx.numw), dtype=torch.float64, device="cuda")
        mo = torch.empty_like(m)
        ctx.forward_rf_full_device(m.data_ptr(), ncol, so.data_ptr(), rf.data_ptr(), mo.data_ptr(), hydrostatic=True)
        torch.cuda.synchronize()
        return so.cpu().numpy(), rf.cpu().numpy()

    s0, r0 = run()
    params = [(25.0, 0.0), (25.0, 0.0)]
    for r, (sg, w0) in enumerate(params):
        ctx.lsf_gaussian(r, sg, w0)
    ks, valid = _kernels(reg, params)
    s1, r1 = run()
    np.testing.assert_allclose(s1, lo.convolve(s0, nw, ks, valid), **TOL)
    rr = r0.reshape(ncol, 6, nz, 4, ctx.numw)
    np.testing.assert_allclose(r1.reshape(rr.shape), lo.convolve(rr, nw, ks, valid), **TOL)


def test_inversion_with_lsf(fz, orc):
    """Observations synthesised with the LSF plus 1e-3 noise: the chi2 of
    the true model (errors mode) is ~1 with the LSF and far above without;
    a short inversion from the perturbed guess reduces chi2 at least 5x."""
    nz, npix = 40, 16
    ctx, reg = _setup(fz, orc, nz)
    ctx.rf_nodes(lmcase.NODES)
    true = fz.atmos.make_columns(npix, nz, seed=23)
    for r in range(2):
        ctx.lsf_gaussian(r, 35.0, 0.0)
    obs, true_he, st = ctx.forward(true, hydrostatic=True)
    assert np.all(st == 0)
    obs = obs + np.random.default_rng(3).normal(0.0, 1e-3, obs.shape)
    opts = fz.LMOpts(maxsteps=5, maxit=20, isigma=1e-3, slots=8)
    _, chi_true, _ = ctx.errors(obs, true_he, hydrostatic=True, opts=opts)
    assert np.median(chi_true) < 1.5
    init = lmcase.initial_guess(true_he, seed=1)
    _, chi_init, _ = ctx.errors(obs, init, hydrostatic=True, opts=opts)
    best, chi, it, st = ctx.invert(obs, init, hydrostatic=True, opts=opts)
    assert np.all(st == 0)
    assert np.median(chi) * 5 < np.median(chi_init)
    ctx.lsf_clear()
    _, chi_nolsf, _ = ctx.errors(obs, true_he, hydrostatic=True, opts=opts)
    assert np.median(chi_nolsf) > 10 * np.median(chi_true)
