"""The launch-shape autotuner.

* Warps per block, grid caps and block sizes change the schedule, not the
  arithmetic: the RF path's outputs are bit-identical for every such shape.
  Sixteen lanes per column in the chemistry chain sum the element terms in
  another order, so those outputs are compared at the synthesis tolerances
  (I 1e-5 relative, Q/U/V 1e-6 I_c) and the node Jacobian at 1e-4 of each
  column's largest entry.
* The inversion's slot count is one of the candidates, and each pixel's
  result does not depend on the pool size (tuned default vs another count).
"""
import numpy as np
import pytest

import lmcase

pytestmark = pytest.mark.gpu


def _ctx(fz, nz):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    return fz.Synthesis(lines, reg, nz=nz)


def test_forward_shapes_do_not_change_results(fz):
    import torch
    nz, ncol = 64, 96
    ctx = _ctx(fz, nz)
    ctx.rf_nodes(lmcase.NODES)
    m = fz.atmos.make_columns(ncol, nz, seed=3)
    ctx.tune(chain_warps=4, chain_lanes=32, chemder_blocks_per_sm=32, opac_rf_threads=256)
    ref = ctx.forward_rf(m, hydrostatic=True)
    d = torch.from_numpy(m).cuda()
    t = ctx.autotune_forward(d.data_ptr(), ncol, hydrostatic=True)
    assert t["chain_warps"] in (1, 2, 4) and t["chain_lanes"] in (0, 32, 16)
    assert t["chemder_blocks_per_sm"] in (0, 8, 16, 32, 64)
    assert t["opac_rf_threads"] in (64, 128, 256)
    assert t["chain_ms"] > 0 and t["chemder_ms"] > 0 and t["opac_rf_ms"] > 0
    for shapes in ({}, dict(chain_warps=1, chain_lanes=32, chemder_blocks_per_sm=0, opac_rf_threads=64),
                   dict(chain_warps=2, chain_lanes=16, chemder_blocks_per_sm=8, opac_rf_threads=128),
                   dict(chain_warps=4, chain_lanes=16)):
        if shapes:
            ctx.tune(**shapes)
        out = ctx.forward_rf(m, hydrostatic=True)
        if ctx.tune()["chain_lanes"] == 32:
            for a, b in zip(ref, out):
                assert np.array_equal(a, b)
        else:
            syn, jac, mo, st = out
            assert np.all(st == 0)
            assert np.max(np.abs(syn[:, 0] - ref[0][:, 0]) / np.abs(ref[0][:, 0])) < 1e-5
            assert np.max(np.abs(syn[:, 1:] - ref[0][:, 1:])) < 1e-6
            scale = np.abs(ref[1]).max(axis=2, keepdims=True)
            assert np.max(np.abs(jac - ref[1]) / scale) < 1e-4
            assert np.allclose(mo, ref[2], rtol=2e-6, atol=0)
    with pytest.raises(fz.FzError):
        ctx.tune(opac_rf_threads=96)


def test_lm_slots_autotune(fz):
    import torch
    nz, npix = 48, 256
    ctx = _ctx(fz, nz)
    ctx.rf_nodes(lmcase.NODES)
    true = fz.atmos.make_columns(npix, nz, seed=77)
    obs, _, _ = ctx.forward(true, hydrostatic=True)
    obs = obs + np.random.default_rng(2).normal(0.0, 1e-3, obs.shape)
    init = lmcase.initial_guess(true)
    opts = fz.LMOpts(maxsteps=5, maxit=20, isigma=1e-3, dchi2=1e-3)
    d_obs = torch.from_numpy(np.ascontiguousarray(obs)).cuda()
    d_init = torch.from_numpy(np.ascontiguousarray(init, dtype=np.float32)).cuda()
    t = ctx.autotune_lm(npix, d_obs.data_ptr(), d_init.data_ptr(), candidates=(64, 128, 256), opts=opts)
    assert t["lm_slots"] in (64, 128, 256) and t["lm_pixels_per_s"] > 0
    assert ctx.tune()["lm_slots"] == t["lm_slots"]
    _, chi_a, _, st_a = ctx.invert(obs, init, hydrostatic=True, opts=opts)
    other = 64 if t["lm_slots"] != 64 else 256     # each pixel's iterations do not depend on the pool
    _, chi_b, _, st_b = ctx.invert(obs, init, hydrostatic=True,
                                   opts=fz.LMOpts(maxsteps=5, maxit=20, isigma=1e-3, dchi2=1e-3, slots=other))
    assert np.all(st_a == 0) and np.all(st_b == 0)
    assert np.array_equal(chi_a, chi_b)
