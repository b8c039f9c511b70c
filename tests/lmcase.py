"""Shared inversion test case: true atmospheres, their synthetic observations
and a perturbed initial guess (TEST INFRASTRUCTURE)."""
import numpy as np

NODES = {1: 5, 4: 2, 5: 2, 6: 2, 7: 2}   # T 5, Bx, By, Bz, v_z 2 each: NP = 13


def initial_guess(true, seed=0):
    """The true model with T offset by ~200 K, the field halved and v_z zeroed."""
    rng = np.random.default_rng(seed)
    m = true.copy()
    m[:, 0] += (150.0 + 100.0 * rng.random((m.shape[0], 1))).astype(np.float32)
    m[:, 5:8] *= 0.5
    m[:, 10] = 0.0
    return m.astype(np.float32)


def oracle_forward_rf(orc, lines, reg, g, he, nodes=None):
    nodes = nodes or NODES

    def f(models):
        syn, jac, mo, st = orc.forward_rf(lines, reg, g, models, nodes, hydrostatic=he)
        n = syn.shape[0]
        return syn.reshape(n, -1), np.transpose(jac, (0, 2, 1)), mo, st
    return f
