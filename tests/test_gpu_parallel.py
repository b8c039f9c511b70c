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


@pytest.mark.parametrize("nx,world", [(6, 2), (7, 3)])
def test_set_tau_shards_equal_whole_field(fz, orc, nx, world):
    """SET_TAU's assists on shards of a field (fz_set_tau_shard_device), the
    field sum and maxima exchanged between the shards by the host threads
    that run them (each shard its own context and stream; no kernel waits
    for another), equal the whole field's fz_set_tau_device bit for bit."""
    import threading

    import torch
    from firtez_dz_b200 import parallel
    ny, nz = 5, 32
    ctx, lines, reg, g = _ctx(fz, orc, nz)
    numw = ctx.numw
    true = fz.atmos.make_columns(nx * ny, nz, seed=61)
    obs, _, _ = ctx.forward(true, hydrostatic=True)
    obs = obs.reshape(nx * ny, -1) + np.random.default_rng(2).normal(0.0, 1e-3, (nx * ny, 4 * numw))
    from firtez_dz_b200 import warmstart as ws
    base = ws.default_models(nx * ny, nz)
    assist = ("temp", "bvec", "vlos")
    d_obs = torch.from_numpy(obs).cuda()
    want = torch.from_numpy(base.copy()).cuda()
    ctx.set_tau_device(nx, ny, d_obs.data_ptr(), want.data_ptr(), assist)
    torch.cuda.synchronize()
    # the host-side exchange of the threads: field_reduce's semantics
    spans = parallel.split(nx, world)
    bar = threading.Barrier(world)
    box = {}

    def reducer(r):
        def fn(kind, data, n, nxr):
            if kind == 0:
                box[("p", r)] = np.array(data[:nxr * n]).reshape(nxr, n)
                bar.wait()
                tot = np.zeros(n)
                for q in range(world):
                    for row in box[("p", q)]:
                        tot = tot + row
                data[:n] = tot
            else:
                box[("m", r)] = np.array(data[:3])
                bar.wait()
                data[:3] = np.max([box[("m", q)] for q in range(world)], axis=0)
            bar.wait()
            return 0
        return fn

    ctxs = [_ctx(fz, orc, nz)[0] for _ in range(world)]
    outs, errs = [], []
    for r, (x0, x1) in enumerate(spans):
        outs.append(torch.from_numpy(base[x0 * ny:x1 * ny].copy()).cuda())

    def run(r):
        try:
            x0, x1 = spans[r]
            ctxs[r].set_tau_shard_device(x1 - x0, ny, d_obs[x0 * ny:].data_ptr(), outs[r].data_ptr(), assist,
                                         reducer(r))
        except Exception as e:   # noqa: BLE001
            errs.append(e)
            bar.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errs, errs
    torch.cuda.synchronize()
    got = torch.cat(outs).cpu().numpy()
    np.testing.assert_array_equal(got, want.cpu().numpy())
