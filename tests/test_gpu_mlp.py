"""The warm-start network on the GPU.

* Forward and gradients of the BF16 kernels against the FP64 oracle
  (oracle/mlp_oracle.py) evaluated on the same bf16-rounded operands; the GPU
  also keeps the activations and dL/dz in bf16 between layers, so each
  layer's gradient is compared in relative L2 norm:
      |g_gpu - g_oracle| <= 3e-2 |g_oracle|,  outputs within 1e-2.
* Per-output loss weights against the loss and bias gradient in numpy.
* Training reduces the loss.
* The gain over the method without it: LM started from the network's
  prediction reaches a lower median chi2 in fewer iterations than LM from
  the default guess, on held-out seeded pixels.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402
import lmcase  # noqa: E402

pytestmark = pytest.mark.gpu

DIMS = (896, 1024, 1024, 512, 13)


def _layers(flat, dims):
    out, o = [], 0
    for i in range(len(dims) - 1):
        n = dims[i] * dims[i + 1] + dims[i + 1]
        out.append(flat[o:o + n])
        o += n
    return out


def test_forward_and_gradients_match_oracle(fz):
    import torch
    from firtez_dz_b200 import warmstart as ws
    net = ws.MLP(DIMS, seed=3)
    assert net.nparams == 2499597
    rng = np.random.default_rng(4)
    n = 256
    x = rng.standard_normal((n, DIMS[0])).astype(np.float32)
    t = rng.standard_normal((n, DIMS[-1])).astype(np.float32)
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    y = torch.empty((n, DIMS[-1]), dtype=torch.float32, device="cuda")
    net.forward_device(n, dx.data_ptr(), y.data_ptr())
    p = net.get_params()
    yo, _ = mo.forward(p, DIMS, x)
    yg = y.cpu().numpy()
    assert np.linalg.norm(yg - yo) <= 1e-2 * np.linalg.norm(yo)
    loss = net.grad_device(n, dx.data_ptr(), dt.data_ptr())
    g = net.get_params(grads=True)
    lo, go = mo.loss_and_grad(p, DIMS, x, t)
    assert abs(loss - lo) <= 1e-2 * lo
    for a, b in zip(_layers(g, DIMS), _layers(go, DIMS)):
        assert np.linalg.norm(a - b) <= 3e-2 * np.linalg.norm(b)


def test_loss_weights(fz):
    """fz_mlp_set_loss_weights: the loss is sum_j w_j (y_j - t_j)^2 / (n
    nout) of the network's own outputs, and the last layer's bias gradient
    2 w_j (y_j - t_j) / (n nout) summed over rows; equal weights give the
    plain loss; a weight vector of the wrong length or a negative weight is
    refused."""
    import torch
    from firtez_dz_b200 import warmstart as ws
    net = ws.MLP(DIMS, seed=5)
    rng = np.random.default_rng(6)
    n = 256
    x = rng.standard_normal((n, DIMS[0])).astype(np.float32)
    t = rng.standard_normal((n, DIMS[-1])).astype(np.float32)
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    y = torch.empty((n, DIMS[-1]), dtype=torch.float32, device="cuda")
    net.forward_device(n, dx.data_ptr(), y.data_ptr())
    d = y.cpu().numpy().astype(np.float64) - t
    w = rng.uniform(0.0, 3.0, DIMS[-1]).astype(np.float32)
    net.set_loss_weights(w)
    loss_w = net.grad_device(n, dx.data_ptr(), dt.data_ptr())
    gb = net.get_params(grads=True)[-DIMS[-1]:]
    ref = float(np.mean(d * d * w[None, :]))
    assert abs(loss_w - ref) <= 1e-5 * ref
    gref = (2.0 * d * w[None, :]).sum(axis=0) / d.size
    assert np.linalg.norm(gb - gref) <= 2e-2 * np.linalg.norm(gref)   # dL/dy rounded to bf16
    net.set_loss_weights(np.ones(DIMS[-1]))
    loss_1 = net.grad_device(n, dx.data_ptr(), dt.data_ptr())
    net.set_loss_weights(None)
    loss_0 = net.grad_device(n, dx.data_ptr(), dt.data_ptr())
    # the blocks' partial sums meet in atomics, in no fixed order
    assert abs(loss_1 - loss_0) <= 1e-6 * loss_0 and abs(loss_0 - float(np.mean(d * d))) <= 1e-5 * loss_0
    with pytest.raises(fz.FzError):
        net.set_loss_weights(np.ones(DIMS[-1] - 1))
    with pytest.raises(fz.FzError):
        net.set_loss_weights(-np.ones(DIMS[-1]))


def test_training_reduces_loss(fz):
    import torch
    from firtez_dz_b200 import warmstart as ws
    rng = np.random.default_rng(1)
    n, d = 16384, 64
    x = rng.standard_normal((n, d)).astype(np.float32)
    a = rng.standard_normal((d, 5)) / np.sqrt(d)
    t = np.tanh(x @ a).astype(np.float32)
    net = ws.MLP((d, 256, 256, 5), seed=2)
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    first = net.train_device(n, dx.data_ptr(), dt.data_ptr(), batch=256, epochs=1, lr=1e-3, seed=1)
    last = net.train_device(n, dx.data_ptr(), dt.data_ptr(), batch=256, epochs=8, lr=1e-3, seed=2)
    assert last < 0.2 * first, (first, last)


def test_warm_start_beats_default_guess(fz):
    from firtez_dz_b200 import warmstart as ws
    nz = 64
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    ctx = fz.Synthesis(lines, reg, nz=nz)
    warm = ws.WarmStart(nz, lmcase.NODES, ctx.numw, seed=5)
    x, t = warm.make_training_set(ctx, 131072, seed=11, noise=1e-3)
    loss = warm.fit(x, t, epochs=6, batch=1024, lr=1e-3)
    assert loss < 0.5   # normalised targets: well below the variance 1
    npix = 96
    true = fz.atmos.make_columns(npix, nz, seed=424242)
    obs, true_he, _ = ctx.forward(true, hydrostatic=True)
    obs = obs + np.random.default_rng(9).normal(0.0, 1e-3, obs.shape)
    ctx.rf_nodes(lmcase.NODES)
    opts = fz.LMOpts(maxsteps=5, maxit=40, isigma=1e-3, dchi2=1e-3)
    _, chi_p, it_p, st_p = ctx.invert(obs, ws.default_models(npix, nz), hydrostatic=True, opts=opts)
    _, chi_w, it_w, st_w = ctx.invert(obs, warm.initial_models(obs), hydrostatic=True, opts=opts)
    assert np.all(st_p == 0) and np.all(st_w == 0)
    assert np.median(chi_w) < np.median(chi_p), (np.median(chi_w), np.median(chi_p))
    assert it_w.mean() <= it_p.mean() + 1.0
    # the fused path: fz_warm_start_device (standardisation inside the bf16
    # conversion, node expansion kernel) gives the models of the host glue
    # above to FP32 rounding, and fz_invert_warm (observations cross once)
    # the inversion of those models
    import torch
    d_obs = torch.from_numpy(obs.reshape(npix, -1)).cuda()
    d_base = torch.from_numpy(ws.default_models(1, nz)[0]).cuda()
    d_out = torch.empty((npix, 13, nz), dtype=torch.float32, device="cuda")
    warm.models_device(ctx, npix, d_obs.data_ptr(), d_base.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    glue = warm.initial_models(obs)
    fused = d_out.cpu().numpy()
    for row in (0, 5, 6, 7, 10):
        scale = np.maximum(np.abs(glue[:, row]).max(axis=1, keepdims=True), 1.0)
        assert np.max(np.abs(fused[:, row] - glue[:, row]) / scale) < 1e-4, row
    assert np.array_equal(np.delete(fused, (0, 5, 6, 7, 10), axis=1), np.delete(glue, (0, 5, 6, 7, 10), axis=1))
    mo_f, chi_f, it_f, st_f = ctx.invert_warm(obs, warm, opts=opts)
    mo_g, chi_g, it_g, st_g = ctx.invert(obs, fused, hydrostatic=True, opts=opts)
    assert np.all(st_f == 0)
    assert np.array_equal(chi_f, chi_g) and np.array_equal(it_f, it_g) and np.array_equal(mo_f, mo_g)


def test_refined_targets(fz):
    """WarmStart.refine_targets: each training pixel is inverted from the
    model of its true node values and its target becomes the node values of
    the inversion's best model.  Those nodes reproduce that model (their
    expansion's chi2 is the inversion's best chi2, never above the true
    nodes' chi2), and a network trained on them starts the held-out pixels
    at a lower median chi2 than the same network trained on the true node
    averages."""
    import torch
    from firtez_dz_b200 import warmstart as ws
    nz, ntrain = 64, 131072
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    ctx = fz.Synthesis(lines, reg, nz=nz)
    ctx.rf_nodes(lmcase.NODES)
    one = fz.LMOpts(maxsteps=5, maxit=1, isigma=1e-3, dchi2=1e-3)
    refine = fz.LMOpts(maxsteps=2, maxit=15, isigma=1e-3, dchi2=1e-3, slots=32768)
    nets = {}
    for kind in ("true", "refined"):
        warm = ws.WarmStart(nz, lmcase.NODES, ctx.numw, seed=5)
        x, t = warm.make_training_set(ctx, ntrain, seed=11, noise=1e-3)
        if kind == "refined":
            t_true = t[:256].double().cpu().numpy() * warm.tsd + warm.tmu
            t, info = warm.refine_targets(ctx, x, t, refine)
            assert info["pixels"] == ntrain and 1.0 <= info["mean_iterations"] <= 15.0
            # the first 256 training pixels: the refined nodes' models against
            # the true nodes' models on the same observations
            obs = (x[:256].double() * warm.xsd.double() + warm.xmu.double()).cpu().numpy().reshape(256, 4, -1)
            base = torch.from_numpy(ws.default_models(1, nz)[0])
            t_ref = t[:256].double().cpu().numpy() * warm.tsd + warm.tmu
            m_true = warm.expand_nodes(torch.from_numpy(t_true), base).numpy()
            m_ref = warm.expand_nodes(torch.from_numpy(t_ref), base).numpy()
            _, c_true, _, s1 = ctx.invert(obs, m_true, hydrostatic=True, opts=one)
            _, c_ref, _, s2 = ctx.invert(obs, m_ref, hydrostatic=True, opts=one)
            best_lm = ctx.invert(obs, m_true, hydrostatic=True, opts=refine)[1]
            assert np.all(s1 == 0) and np.all(s2 == 0)
            # the targets are kept standardised in float32, so the refined
            # nodes reproduce the best model to that rounding
            q = np.quantile(c_ref / c_true, [0.5, 0.9, 0.99, 1.0])
            assert q[2] <= 1.0 + 1e-4, q
            assert np.median(np.abs(c_ref / best_lm - 1.0)) < 1e-3, np.quantile(c_ref / best_lm, [0.01, 0.5, 0.99])
        warm.fit(x, t, epochs=6, batch=1024, lr=1e-3)
        del x
        nets[kind] = warm
    npix = 512
    true = fz.atmos.make_columns(npix, nz, seed=424243)
    obs, _, _ = ctx.forward(true, hydrostatic=True)
    obs = obs + np.random.default_rng(19).normal(0.0, 1e-3, obs.shape)
    med = {k: np.median(ctx.invert(obs, w.initial_models(obs), hydrostatic=True, opts=one)[1])
           for k, w in nets.items()}
    assert med["refined"] < med["true"], med

