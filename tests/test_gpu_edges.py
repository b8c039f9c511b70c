"""Edge cases of the GPU path against the oracle (same tolerances as the
main parity tests: Stokes I 1e-5 relative, Q/U/V 1e-6 I_c, node Jacobian
2e-4 of each column's largest entry).

* Ragged sizes: one column and three columns, 9 heights, regions of 7 and
  33 wavelengths (thread blocks with idle lanes, a region boundary inside a
  warp), with and without hydrostatic equilibrium.
* A pixel count below the slot count, and a single pixel.
* Empty batches are rejected; a column with a non-finite temperature gets a
  non-zero status while the other columns of the same call are unaffected.
"""
import numpy as np
import pytest

import lmcase

pytestmark = pytest.mark.gpu

RF_TOL = 2e-4


def _setup(fz, orc, section):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(section, lines)
    g, _ = orc.gain(lines, reg)
    return lines, reg, g


@pytest.mark.parametrize("ncol", [1, 3])
@pytest.mark.parametrize("he", [True, False])
def test_ragged_sizes_match_oracle(fz, orc, ncol, he):
    nz = 9
    lines, reg, g = _setup(fz, orc, "1 7 -64.5 21.5\n2 33 -344.0 21.5\n")
    m = fz.atmos.make_columns(ncol, nz, seed=41)
    if not he:
        _, m, _ = orc.forward(lines, reg, g, m, hydrostatic=True)
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    assert ctx.numw == 40
    syn, mo, st = ctx.forward(m, hydrostatic=he)
    ref, mref, sref = orc.forward(lines, reg, g, m, hydrostatic=he)
    assert np.all(st == 0) and np.all(sref == 0)
    assert np.max(np.abs(syn[:, 0] / ref[:, 0] - 1)) < 1e-5
    assert np.max(np.abs(syn[:, 1:] - ref[:, 1:])) < 1e-6
    nodes = {1: 3, 4: 1, 5: 1, 6: 1, 7: 1}
    ctx.rf_nodes(nodes)
    _, jac, _, st2 = ctx.forward_rf(m, hydrostatic=he)
    _, ojac, _, _ = orc.forward_rf(lines, reg, g, m, nodes, hydrostatic=he)
    assert np.all(st2 == 0)
    scale = np.abs(ojac).max(axis=2, keepdims=True)
    assert np.all(scale > 0)
    assert np.max(np.abs(jac - ojac) / scale) <= RF_TOL


@pytest.mark.parametrize("npix,slots", [(1, 4), (3, 8)])
def test_few_pixels_and_spare_slots(fz, orc, npix, slots):
    nz = 32
    lines, reg, g = _setup(fz, orc, fz.atmos.lines_section(2))
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    true = fz.atmos.make_columns(npix, nz, seed=8)
    obs, true_he, _ = ctx.forward(true, hydrostatic=True)
    init = lmcase.initial_guess(true_he, seed=3)
    syn0, _, _ = ctx.forward(init, hydrostatic=True)
    ctx.rf_nodes(lmcase.NODES)
    opts = fz.LMOpts(maxsteps=5, maxit=20, isigma=1e-3, dchi2=1e-3, slots=slots)
    best, chi, it, st = ctx.invert(obs, init, hydrostatic=True, opts=opts)
    assert best.shape == (npix, 13, nz) and np.all(st == 0)
    assert np.all(it >= 1) and np.all(it <= 20)
    w = 1.0 / (1e-3 ** 2)
    chi0 = np.sum((obs - syn0) ** 2, axis=(1, 2)) * w / (4 * ctx.numw)
    assert np.all(chi < chi0)


def test_empty_batches_are_rejected(fz, orc):
    lines, reg, g = _setup(fz, orc, fz.atmos.lines_section(2))
    ctx = fz.Synthesis(lines, reg, nz=16, gain=g)
    with pytest.raises((fz.FzError, ValueError)):
        ctx.forward(np.zeros((0, 13, 16), dtype=np.float32))
    ctx.rf_nodes({1: 2})
    with pytest.raises((fz.FzError, ValueError)):
        ctx.invert(np.zeros((0, 4, ctx.numw)), np.zeros((0, 13, 16), dtype=np.float32))


def test_non_finite_column_is_flagged_alone(fz, orc):
    nz, ncol = 24, 5
    lines, reg, g = _setup(fz, orc, fz.atmos.lines_section(2))
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    m = fz.atmos.make_columns(ncol, nz, seed=19)
    good, _, stg = ctx.forward(m, hydrostatic=False)
    bad = m.copy()
    bad[2, 0, nz // 2] = np.nan
    syn, _, st = ctx.forward(bad, hydrostatic=False)
    assert np.all(stg == 0)
    assert st[2] != 0
    keep = [0, 1, 3, 4]
    assert np.all(st[keep] == 0)
    np.testing.assert_array_equal(syn[keep], good[keep])
