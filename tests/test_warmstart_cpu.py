"""Node-space helpers of the warm start on CPU tensors (no network is
built): expand_nodes is expand() on tensors, and fit_nodes -- the
least-squares node values whose expansion reproduces a model, which
refine_targets uses to turn an inversion's best model into a training
target -- inverts it to the float32 rounding of the models."""
import numpy as np

import lmcase


def test_node_expansion_round_trip(fz, monkeypatch):
    import torch
    from firtez_dz_b200 import warmstart as ws
    monkeypatch.setattr(ws, "MLP", lambda *a, **k: None)
    nz, npix = 96, 7
    warm = ws.WarmStart(nz, lmcase.NODES, 224)
    base1 = ws.default_models(1, nz)
    bases = np.repeat(base1, npix, axis=0)
    n0 = warm.targets(bases)
    scale = np.array([300.0] * 5 + [50.0] * 6 + [0.5] * 2)
    nodes = n0 + np.random.default_rng(3).normal(size=n0.shape) * scale
    m = warm.expand_nodes(torch.from_numpy(nodes), torch.from_numpy(base1[0]))
    assert np.array_equal(m.numpy(), warm.expand(nodes, bases))
    back = warm.fit_nodes(m, torch.from_numpy(base1[0])).numpy()
    j = 0
    for p, row in warm.params:
        nj = warm.nodes[p]
        tol = 8 * np.finfo(np.float32).eps * np.abs(m[:, row].numpy()).max()
        assert np.all(np.abs(back[:, j:j + nj] - nodes[:, j:j + nj]) <= tol), (p, tol)
        j += nj
