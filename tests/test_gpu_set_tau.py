"""SET_TAU's assists on the GPU against the oracle's restatement
(oracle/tau_oracle.py) on a 9 x 7 field: B and v_z (constant in height)
within 2e-6 relative of the field scale (the projections' FP64 sums differ
in order), T within 1e-3 K, Pg within 1 ulp; with T or Pg the derived rows
come from the plain synthesis of the assisted model (checked against the
oracle's synthesis of the same model).  Inside the cycle loop the assists
run at the start of a cycle whose Pg is not free."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import lmcase  # noqa: E402
import tau_oracle as to  # noqa: E402

pytestmark = pytest.mark.gpu


def _field(fz, orc, nz, nx, ny, seed):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    true = fz.atmos.make_columns(nx * ny, nz, seed=seed)
    obs, true_he, _ = orc.forward(lines, reg, g, true, hydrostatic=True)
    obs = obs + np.random.default_rng(seed).normal(0.0, 1e-3, obs.shape)
    l0 = float(ctx.lines["l0"][int(reg["line"][0][0])])
    return ctx, lines, reg, g, obs, true_he, int(reg["numwave"][0]), l0


@pytest.mark.parametrize("he", [False, True])
@pytest.mark.parametrize("assist", [("bvec",), ("vlos",), ("bvec", "vlos"), ("temp",), ("pgas",),
                                    ("temp", "pgas", "bvec", "vlos")])
def test_set_tau_matches_oracle(fz, orc, assist, he):
    nx, ny, nz = 9, 7, 40
    ctx, lines, reg, g, obs, true_he, n1, l0 = _field(fz, orc, nz, nx, ny, 5)
    init = lmcase.initial_guess(true_he, seed=2)
    got = ctx.set_tau(obs, init, nx, ny, assist, hydrostatic=he)
    ref = to.set_tau(obs, init, nx, ny, n1, l0, set(assist))
    for row in (5, 6, 7, 10):
        scale = np.max(np.abs(ref[:, row])) + 1e-30
        np.testing.assert_allclose(got[:, row], ref[:, row], rtol=0, atol=2e-6 * scale)
    np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=0, atol=1e-3)
    if "temp" in assist or "pgas" in assist:
        # the derived rows (and, hydrostatic, Pg integrated from the anchor
        # ITZ the assists marked) are the plain synthesis' of the assisted
        # model: the oracle's of the oracle's assisted model
        _, mo, st = orc.forward(lines, reg, g, ref, hydrostatic=2 if he else 0)
        assert np.all(st == 0)
        for row in (1, 2, 3, 4):
            np.testing.assert_allclose(got[:, row], mo[:, row], rtol=5e-6, atol=0)
        np.testing.assert_allclose(got[:, 11], mo[:, 11], rtol=0, atol=1e-5)
    else:
        np.testing.assert_array_equal(got[:, [0, 1, 2, 3, 4, 11]], init[:, [0, 1, 2, 3, 4, 11]])


def test_set_tau_in_cycles(fz, orc):
    """invert_cycles with the B and v_z assists equals SET_TAU, SMOOTHING_B
    and the inversion run one after the other; progressive runs them in the
    first cycle only."""
    nx, ny, nz = 6, 4, 40
    ctx, lines, reg, g, obs, true_he, n1, l0 = _field(fz, orc, nz, nx, ny, 8)
    init = lmcase.initial_guess(true_he, seed=4)
    nodes = lmcase.NODES
    opts = fz.LMOpts(maxsteps=5, maxit=8, isigma=1e-3, slots=8, assist=("bvec", "vlos"))
    mod, chi, it, st = ctx.invert_cycles(obs, init, nx, ny, [nodes], hydrostatic=True, opts=opts)
    ctx.rf_nodes(nodes)
    m = ctx.set_tau(obs, init, nx, ny, ("bvec", "vlos"))
    m = ctx.smooth(m, nx, ny)
    opts2 = fz.LMOpts(maxsteps=5, maxit=8, isigma=1e-3, slots=8)
    best, chi2, _, _ = ctx.invert(obs, m, hydrostatic=True, opts=opts2)
    np.testing.assert_array_equal(chi, chi2)
    assert np.all(st == 0)
