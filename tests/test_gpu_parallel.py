"""The shard mode of SMOOTHING_B on the GPU (fz_smooth_shard_device): shards
of a field with their neighbours' halo columns attached, smoothed one by one,
give the whole field's SMOOTHING_B bit for bit (the exchange itself is
covered by the gloo tests on CPU); and FieldShard's cycle loop on one rank
equals fz_invert_cycles_device."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import lmcase  # noqa: E402

pytestmark = pytest.mark.gpu


def _ctx(fz, orc, nz):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    return fz.Synthesis(lines, reg, nz=nz, gain=g), lines, reg, g


@pytest.mark.parametrize("nx,world", [(7, 2), (9, 4), (4, 2), (6, 3)])
def test_smooth_shards_equal_whole_field(fz, orc, nx, world):
    import torch
    from firtez_dz_b200 import parallel
    ny, nz = 5, 16
    ctx = _ctx(fz, orc, nz)[0]
    ctx.rf_nodes({1: 2, 4: 1, 6: 1, 7: 1})
    full = np.random.default_rng(nx).standard_normal((nx * ny, 13, nz)).astype(np.float32) * 100
    want = torch.from_numpy(full.copy()).cuda()
    ctx.smooth_device(want.data_ptr(), nx, ny)
    torch.cuda.synchronize()
    for x0, x1 in parallel.split(nx, world):
        a, b = max(0, x0 - 1), min(nx, x1 + 1)
        ext = torch.from_numpy(full[a * ny:b * ny].copy()).cuda()
        ctx.smooth_shard_device(ext.data_ptr(), b - a, ny, a, nx)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(ext[(x0 - a) * ny:(x1 - a) * ny].cpu().numpy(),
                                      want[x0 * ny:x1 * ny].cpu().numpy())


def test_field_shard_cycles_one_rank(fz, orc):
    import torch
    from firtez_dz_b200 import parallel
    nx, ny, nz = 5, 4, 40
    ctx, lines, reg, g = _ctx(fz, orc, nz)
    true = fz.atmos.make_columns(nx * ny, nz, seed=12)
    obs, true_he, _ = orc.forward(lines, reg, g, true, hydrostatic=True)
    init = lmcase.initial_guess(true_he, seed=3)
    cycles = [{1: 2, 6: 1, 7: 1}, lmcase.NODES]
    opts = fz.LMOpts(maxsteps=5, maxit=10, isigma=1e-3, slots=8)
    mod, chi, it, st = ctx.invert_cycles(obs, init, nx, ny, cycles, hydrostatic=True, opts=opts)
    sh = parallel.FieldShard(nx, ny, 0, 1)
    d_obs = torch.from_numpy(np.ascontiguousarray(obs)).cuda()
    d_m = torch.from_numpy(init.copy()).cuda()
    chi2, it2, st2 = sh.invert_cycles(ctx, d_obs, d_m, cycles, hydrostatic=True, opts=opts)
    np.testing.assert_array_equal(chi2.cpu().numpy(), chi)
    np.testing.assert_array_equal(it2.cpu().numpy(), it)
    np.testing.assert_array_equal(d_m.cpu().numpy(), mod)
