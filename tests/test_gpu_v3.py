"""v3 files with the GPU: the layout kernels against the oracle's numpy
restatement (oracle/v3_oracle.py; pure data movement, bit-exact), and the
drop-in flows of the reference's test cases on files: a model file
synthesised into a profile file (tests/test_syn1), the full-height response
functions into an RF file (tests/test_rf), and a profile file read as the
inversion's observations with the inverted models written back as a model
file (tests/test_inv1)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import lmcase  # noqa: E402
import v3_oracle as vo  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def v3(fz):
    from firtez_dz_b200 import v3io
    return v3io


def _ctx(fz, orc, nz):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    return fz.Synthesis(lines, reg, nz=nz, gain=g), lines, reg, g


@pytest.mark.parametrize("nx,ny,nz,nw", [(5, 3, 7, 9), (1, 1, 256, 224), (17, 9, 128, 224)])
def test_layout_kernels_match_oracle(fz, v3, nx, ny, nz, nw):
    import torch
    rng = np.random.default_rng(nx * 100 + ny)
    cubes = rng.standard_normal((13, nx, ny, nz)).astype(np.float32)
    d_model = v3.model_from_cubes_device(torch.from_numpy(cubes).cuda())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_model.cpu().numpy(), vo.model_from_cubes(cubes))
    model = rng.standard_normal((nx * ny, 13, nz)).astype(np.float32)
    x = rng.uniform(0, 1e4, nx)
    y = rng.uniform(0, 1e4, ny)
    d_c = v3.cubes_from_model_device(torch.from_numpy(model).cuda(), nx, ny, x, y)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_c.cpu().numpy(), vo.cubes_from_model(model, nx, ny, x, y))
    st = rng.standard_normal((nx, ny, nw, 4)).astype(np.float32)
    d_obs = v3.obs_from_stokes_device(torch.from_numpy(st).cuda())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_obs.cpu().numpy(), vo.obs_from_stokes(st))
    syn = rng.standard_normal((nx * ny, 4, nw))
    d_st = v3.stokes_from_syn_device(torch.from_numpy(syn).cuda(), nx, ny)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_st.cpu().numpy(), vo.stokes_from_syn(syn, nx, ny))
    if nx * ny * nz * nw <= 200000:
        rf = rng.standard_normal((nx * ny, 6, nz, 4 * nw)).astype(np.float32)
        d_rf = v3.rf_file_layout_device(torch.from_numpy(rf).cuda(), nx, ny)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_rf.cpu().numpy(), vo.rf_payload(rf, nx, ny))


def test_model_file_synthesis_to_profile_file(fz, orc, v3, tmp_path):
    """test_syn1 on files: a 4 x 3 x 48 model file (the columns of the
    synthetic generator, x, y in km) -> the device MODEL -> synthesis ->
    the profile file; the file holds the synthesis rounded to REAL*4, and the
    synthesis matches the oracle's of the same columns (I 1e-5 relative,
    Q/U/V 1e-6 of Ic)."""
    import torch
    nx, ny, nz = 4, 3, 48
    ctx, lines, reg, g = _ctx(fz, orc, nz)
    m = fz.atmos.make_columns(nx * ny, nz, seed=8)
    x, y = 16.0 * np.arange(nx), 16.0 * np.arange(ny)
    cubes = vo.cubes_from_model(m, nx, ny, x, y)
    src = tmp_path / "model.bin"
    v3.write_model(src, cubes)
    d_model = v3.model_from_cubes_device(torch.from_numpy(v3.read_model(src)).cuda())
    d_syn = torch.empty((nx * ny, 4, ctx.numw), dtype=torch.float64, device="cuda")
    d_mo = torch.empty_like(d_model)
    ctx.forward_device(d_model.data_ptr(), nx * ny, d_syn.data_ptr(), d_mo.data_ptr(), hydrostatic=False)
    d_st = v3.stokes_from_syn_device(d_syn, nx, ny)
    torch.cuda.synchronize()
    ind = np.ones(ctx.numw)
    wave = np.arange(ctx.numw, dtype=np.float64)
    out = tmp_path / "profiles.bin"
    v3.write_profile(out, ind, wave, d_st.cpu().numpy())
    _, _, st = v3.read_profile(out)
    syn = d_syn.cpu().numpy()
    np.testing.assert_array_equal(st, vo.stokes_from_syn(syn, nx, ny))
    # the file's model equals the generator's in every row the file carries
    # (vx, vy are not in the file; z is the first pixel's column)
    mref = vo.model_from_cubes(cubes)
    np.testing.assert_array_equal(d_model.cpu().numpy(), mref)
    osyn, _, ost = orc.forward(lines, reg, g, mref, hydrostatic=False)
    assert np.all(ost == 0)
    assert np.max(np.abs(syn[:, 0] - osyn[:, 0]) / np.abs(osyn[:, 0])) < 1e-5
    assert np.max(np.abs(syn[:, 1:] - osyn[:, 1:])) < 1e-6


def test_rf_full_to_rf_file(fz, orc, v3, tmp_path):
    """test_rf on files: fz_forward_rf_full's every-height responses of 3 x 2
    columns -> the RF file layout on the device -> the file; read back, the
    payload equals the oracle's layout of the same device output."""
    import torch
    nx, ny, nz = 3, 2, 32
    ctx = _ctx(fz, orc, nz)[0]
    m = torch.from_numpy(fz.atmos.make_columns(nx * ny, nz, seed=5)).cuda()
    nf = 4 * ctx.numw
    rf = torch.empty((nx * ny, 6, nz, nf), dtype=torch.float32, device="cuda")
    so = torch.empty((nx * ny, 4, ctx.numw), dtype=torch.float64, device="cuda")
    mo = torch.empty_like(m)
    ctx.forward_rf_full_device(m.data_ptr(), nx * ny, so.data_ptr(), rf.data_ptr(), mo.data_ptr(), hydrostatic=True)
    d_out = v3.rf_file_layout_device(rf, nx, ny)
    torch.cuda.synchronize()
    z = np.linspace(-500.0, 1500.0, nz)
    out = tmp_path / "rf.bin"
    v3.write_rf(out, z, v3.RF_FULL_LOGV, np.ones(ctx.numw), np.arange(ctx.numw, dtype=np.float64),
                d_out.cpu().numpy())
    zz, logv, _, _, data = v3.read_rf(out)
    assert tuple(logv) == v3.RF_FULL_LOGV
    np.testing.assert_array_equal(data, vo.rf_payload(rf.cpu().numpy(), nx, ny))
    np.testing.assert_array_equal(zz, np.float32(z))


def test_profile_file_inversion_to_model_file(fz, orc, v3, tmp_path):
    """test_inv1 on files: observations written as a v3 profile file (REAL*4,
    as the reference stores them), read into OBS3D on the device, inverted
    from a perturbed guess, the best models written as a model file; the
    inversion from the file's observations equals the inversion from the
    same REAL*4-rounded observations given directly."""
    import torch
    nx, ny, nz = 3, 2, 40
    npix = nx * ny
    ctx, lines, reg, g = _ctx(fz, orc, nz)
    true = fz.atmos.make_columns(npix, nz, seed=13)
    obs, true_he, _ = orc.forward(lines, reg, g, true, hydrostatic=True)
    st = vo.stokes_from_syn(obs, nx, ny)
    pf = tmp_path / "obs.bin"
    v3.write_profile(pf, np.ones(ctx.numw), np.arange(ctx.numw, dtype=np.float64), st)
    _, _, st2 = v3.read_profile(pf)
    d_obs = v3.obs_from_stokes_device(torch.from_numpy(st2).cuda())
    ctx.rf_nodes(lmcase.NODES)
    init = lmcase.initial_guess(true_he, seed=3)
    opts = fz.LMOpts(maxsteps=5, maxit=15, isigma=1e-3, slots=8)
    d_init = torch.from_numpy(init).cuda()
    d_best = torch.empty_like(d_init)
    chi = torch.empty(npix, dtype=torch.float64, device="cuda")
    it = torch.empty(npix, dtype=torch.int32, device="cuda")
    ctx.invert_device(npix, d_obs.data_ptr(), d_init.data_ptr(), d_best.data_ptr(), chi.data_ptr(), it.data_ptr(),
                      opts=opts)
    torch.cuda.synchronize()
    best, chi2, _, _ = ctx.invert(vo.obs_from_stokes(st), init, hydrostatic=True, opts=opts)
    np.testing.assert_array_equal(d_best.cpu().numpy(), best)
    np.testing.assert_array_equal(chi.cpu().numpy(), chi2)
    d_c = v3.cubes_from_model_device(d_best, nx, ny, np.arange(nx) * 16.0, np.arange(ny) * 16.0)
    torch.cuda.synchronize()
    mf = tmp_path / "out_model.bin"
    v3.write_model(mf, d_c.cpu().numpy())
    back = vo.model_from_cubes(v3.read_model(mf))
    rows = [0, 1, 2, 3, 4, 5, 6, 7, 10, 11]
    np.testing.assert_array_equal(back[:, rows], best[:, rows])
