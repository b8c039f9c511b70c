"""GPU synthesis parity against the FP64 CPU oracle, through the C-ABI.

Tolerances (FP32 kernels vs FP64 restatement): Stokes I/Ic within 1e-5
relative, Q/U/V within 1e-6 Ic absolute.  Chemistry and hydrostatic
integration run in FP64 on the GPU; the updated model (rho, Pe, mu, Pg) must
agree to float32 rounding (plus the GET_RHO convergence tolerance).
"""
import numpy as np
import pytest

import fixtures

pytestmark = pytest.mark.gpu

TOL_I = 1e-5
TOL_QUV = 1e-6


def stokes_errors(g, o):
    """max relative error of I, max absolute error of Q/U/V (per column Ic units)."""
    ei = np.max(np.abs(g[:, 0] - o[:, 0]) / np.abs(o[:, 0]))
    eq = np.max(np.abs(g[:, 1:] - o[:, 1:]))
    return ei, eq


@pytest.fixture(scope="module")
def workload(fz, orc):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    return lines, reg


def test_gain_matches_oracle(fz, orc, workload):
    lines, reg = workload
    ctx = fz.Synthesis(lines, reg, nz=96)
    g_gpu = ctx.gain
    g_orc, st = orc.gain(lines, reg)
    assert st == 0
    assert np.max(np.abs(g_gpu / g_orc - 1)) < 2e-7
    assert np.all(g_gpu[:, 3] == -g_gpu[:, 0])


@pytest.mark.parametrize("lanes", [32, 16])
@pytest.mark.parametrize("hydrostatic", [False, True])
def test_synthesis_matches_oracle(fz, orc, workload, hydrostatic, lanes):
    """lanes: lanes per column of the chemistry chain kernel (a launch shape
    the autotuner may pick)."""
    lines, reg = workload
    nz, ncol = 96, 64
    m = fz.atmos.make_columns(ncol, nz, seed=11)
    g, _ = orc.gain(lines, reg)
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    ctx.tune(chain_lanes=lanes)
    syn, mo, st = ctx.forward(m, hydrostatic=hydrostatic)
    ref, mref, sref = orc.forward(lines, reg, g, m, hydrostatic=hydrostatic)
    assert np.all(st == 0) and np.all(sref == 0)
    ei, eq = stokes_errors(syn, ref)
    print("max rel err I %.3e, max abs err QUV %.3e" % (ei, eq))
    assert ei < TOL_I
    assert eq < TOL_QUV
    # updated model: rho, mu (and Pg in hydrostatic mode) to float rounding
    for p in (2, 4) + ((1,) if hydrostatic else ()):
        assert np.max(np.abs(mo[:, p] / mref[:, p] - 1)) < 2e-6, p
    assert np.max(np.abs(mo[:, 11] - mref[:, 11])) < 1e-5     # log tau5


def test_zero_field_gives_zero_polarisation(fz, orc, workload):
    lines, reg = workload
    m = fz.atmos.make_columns(8, 64, seed=5)
    m[:, 5:8] = 0.0
    ctx = fz.Synthesis(lines, reg, nz=64)
    syn, _, st = ctx.forward(m)
    assert np.all(st == 0)
    assert np.all(syn[:, 1:] == 0.0)


def test_reference_fixture_with_blend(fz, orc):
    """test_syn1/test_rf set-up: lines 4,5 blended, 500 points from -700 mA."""
    lines = fz.lines_parse(fixtures.fixture_lines_text())
    reg = fz.regions_from_lines_section("4,5 500 -700.0 5.0", lines)
    m = np.concatenate([fixtures.fixture_model("test_atmos.bin"), fixtures.fixture_model("rf_test_atmos.bin")])
    g, _ = orc.gain(lines, reg)
    ctx = fz.Synthesis(lines, reg, nz=m.shape[2], gain=g)
    syn, mo, st = ctx.forward(m)
    ref, mref, sref = orc.forward(lines, reg, g, m)
    ei, eq = stokes_errors(syn, ref)
    print("fixture: max rel err I %.3e, max abs err QUV %.3e" % (ei, eq))
    assert np.all(syn[0, 1:] == 0.0)          # B = 0 column
    assert ei < TOL_I and eq < TOL_QUV


def test_hydrostatic_from_log_tau5_anchor(fz, orc):
    """Hydrostatic equilibrium anchored at the height of least |log tau5| of
    the input model (HYDRO_TOP off, RK4_INTEGRATION_LOG_LTAUM05): the
    synthesis and the integrated Pg, rho, Pe, mu against the oracle's
    restatement with the same tolerances as the top-anchored mode; Pg at the
    anchor is kept; the anchor at the bottom and at the top columns work."""
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    nz = 64
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    m0 = fz.atmos.make_columns(10, nz, seed=17)
    _, m, st = orc.forward(lines, reg, g, m0, hydrostatic=True)   # a log tau5 row to anchor on
    assert np.all(st == 0)
    m[8, 11, :] = np.linspace(-1.0, 5.0, nz, dtype=np.float32)     # anchor at the bottom
    m[9, 11, :] = np.linspace(-5.0, -1.0, nz, dtype=np.float32)    # anchor at the top
    m[:, 1, :] *= np.float32(1.3)                                   # Pg off equilibrium elsewhere
    syn, mo, st = ctx.forward(m, hydrostatic="ltau")
    osyn, omo, ost = orc.forward(lines, reg, g, m, hydrostatic=2)
    assert np.all(st == 0) and np.all(ost == 0)
    assert np.max(np.abs(syn[:, 0] - osyn[:, 0]) / np.abs(osyn[:, 0])) < 1e-5
    assert np.max(np.abs(syn[:, 1:] - osyn[:, 1:])) < 1e-6
    for p in (1, 2, 3, 4):
        assert np.max(np.abs(mo[:, p] / omo[:, p] - 1)) < 2e-6, p
    iz = np.argmin(np.abs(m[:, 11, :]), axis=1)
    np.testing.assert_allclose(mo[np.arange(10), 1, iz], m[np.arange(10), 1, iz], rtol=1.2e-7)
    with pytest.raises(fz.FzError):
        ctx.rf_nodes({1: 2})
        ctx.forward_rf(m, hydrostatic=2)


@pytest.mark.parametrize("he", [False, True, "ltau"])
def test_model_only_modes(fz, orc, he):
    """MODE t (log tau5 without the synthesis) and MODE h (HE only) give the
    same model rows, bit for bit, as the full synthesis computes them."""
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    nz = 48
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    _, m, _ = orc.forward(lines, reg, g, fz.atmos.make_columns(20, nz, seed=3), hydrostatic=True)
    _, mo, st = ctx.forward(m, hydrostatic=he)
    assert np.all(st == 0)
    mt, st2 = ctx.log_tau5(m, hydrostatic=he)
    assert np.all(st2 == 0)
    np.testing.assert_array_equal(mt, mo)
    if he:
        mh, _ = ctx.hydrostatic(m, mode=he)
        np.testing.assert_array_equal(mh[:, :5], mo[:, :5])
        np.testing.assert_array_equal(mh[:, 5:11], m[:, 5:11])


def test_many_wavelengths(fz, orc):
    """Four spectral regions of 96 wavelengths (NUMW 384, the two-band
    configuration): the synthesis and the node Jacobian (blocks of 512
    threads, one per wavelength) match the oracle with the tolerances of the
    two-line case, and an inversion runs; NUMW 544 (beyond 512) is refused by
    the response-function and inversion entry points with FZ_ERR_LIMIT while
    the synthesis still runs."""
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(4), lines)
    g, _ = orc.gain(lines, reg)
    nz = 40
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    assert ctx.numw == 384
    m = fz.atmos.make_columns(6, nz, seed=2)
    syn, mo, st = ctx.forward(m, hydrostatic=True)
    osyn, omo, ost = orc.forward(lines, reg, g, m, hydrostatic=True)
    assert np.all(st == 0) and np.all(ost == 0)
    assert np.max(np.abs(syn[:, 0] - osyn[:, 0]) / np.abs(osyn[:, 0])) < 1e-5
    assert np.max(np.abs(syn[:, 1:] - osyn[:, 1:])) < 1e-6
    nodes = {1: 3, 4: 1, 5: 1, 6: 2, 7: 2}
    ctx.rf_nodes(nodes)
    rsyn, jac, _, st = ctx.forward_rf(m, hydrostatic=True)
    orsyn, ojac, _, ost = orc.forward_rf(lines, reg, g, m, nodes, hydrostatic=True)
    assert np.all(st == 0) and np.all(ost == 0)
    assert np.max(np.abs(rsyn[:, 0] - orsyn[:, 0]) / np.abs(orsyn[:, 0])) < 1e-5
    scale = np.abs(ojac).max(axis=2)
    rel = np.abs(jac.astype(np.float64) - ojac).max(axis=2) / np.where(scale > 0, scale, 1.0)
    assert rel.max() <= 2e-4, rel.max()
    best, chi, it, st = ctx.invert(syn, m, hydrostatic=True, opts=fz.LMOpts(maxit=3, isigma=1e-3, slots=4))
    assert np.all(st == 0) and np.all(np.isfinite(chi))
    reg5 = fz.regions_from_lines_section(fz.atmos.lines_section(4, nw=136), lines)
    ctx5 = fz.Synthesis(lines, reg5, nz=nz, gain=orc.gain(lines, reg5)[0])
    assert ctx5.numw == 544
    ctx5.forward(m, hydrostatic=True)
    ctx5.rf_nodes({1: 2, 6: 1})
    with pytest.raises(fz.FzError, match="limit"):
        ctx5.forward_rf(m, hydrostatic=True)


def test_four_line_field_at_its_height_count(fz, orc):
    """The four-line workload at its own shape: 160 heights, Fe I 6301.5,
    6302.5, 15648.5 and 15652.9 x 96 wavelengths (NUMW 384, blocks of 512
    threads), |B| up to 4000 G.  Stokes against the oracle with the
    two-line tolerances (I 1e-5 relative, Q/U/V 1e-6 I_c) and the node
    Jacobian of the benchmark's layout (T 5, Bx/By/Bz/v_z 2) within 2e-4 of
    the largest entry of each parameter's node columns."""
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(4), lines)
    g, _ = orc.gain(lines, reg)
    nz = 160
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    assert ctx.numw == 384
    m = fz.atmos.make_columns(4, nz, seed=21, bmax=4000.0)
    syn, mo, st = ctx.forward(m, hydrostatic=True)
    osyn, omo, ost = orc.forward(lines, reg, g, m, hydrostatic=True)
    assert np.all(st == 0) and np.all(ost == 0)
    assert np.max(np.abs(syn[:, 0] - osyn[:, 0]) / np.abs(osyn[:, 0])) < 1e-5
    assert np.max(np.abs(syn[:, 1:] - osyn[:, 1:])) < 1e-6
    nodes = {1: 5, 4: 2, 5: 2, 6: 2, 7: 2}
    ctx.rf_nodes(nodes)
    rsyn, jac, _, st = ctx.forward_rf(m, hydrostatic=True)
    orsyn, ojac, _, ost = orc.forward_rf(lines, reg, g, m, nodes, hydrostatic=True)
    assert np.all(st == 0) and np.all(ost == 0)
    assert np.max(np.abs(rsyn[:, 0] - orsyn[:, 0]) / np.abs(orsyn[:, 0])) < 1e-5
    err = np.abs(jac.astype(np.float64) - ojac).max(axis=2)
    j0 = 0
    for p, nj in sorted(nodes.items()):
        scale = np.abs(ojac[:, j0:j0 + nj]).max(axis=(1, 2))
        assert np.all(scale > 0)
        rel = err[:, j0:j0 + nj].max(axis=1) / scale
        assert rel.max() <= 2e-4, (p, rel.max())
        j0 += nj


@pytest.mark.parametrize("he", [True, False])
def test_small_batch_chain_on_precomputed_saha_factors(fz, workload, he):
    """Batches of at most 1,024 columns run the chemistry chain on Saha
    factors precomputed by k_saha (k_chain_pre); larger ones compute them
    inside the chain.  Both forms (32 lanes a column at these sizes) give
    the same columns bit for bit: 1,024 columns against the first 1,024 of
    1,025."""
    lines, reg = workload
    ctx = fz.Synthesis(lines, reg, nz=64)
    m = fz.atmos.make_columns(1025, 64, seed=77)
    s_big, mo_big, st_big = ctx.forward(m, hydrostatic=he)
    s_small, mo_small, st_small = ctx.forward(m[:1024], hydrostatic=he)
    assert np.all(st_big == 0) and np.all(st_small == 0)
    np.testing.assert_array_equal(s_small, s_big[:1024])
    np.testing.assert_array_equal(mo_small, mo_big[:1024])
    ctx.profile(True)
    ctx.profile_read()
    ctx.forward(m[:8], hydrostatic=he)
    pr = ctx.profile_read()
    ctx.profile(False)
    assert pr["k_saha"][1] == 1 and pr["k_chain_pre"][1] == 1 and pr["k_chain"][1] == 0, pr
