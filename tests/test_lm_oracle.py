"""Pins of the FP64 Levenberg-Marquardt oracle (oracle/lm_oracle.py).

The reference has no golden inversion outputs; the oracle's pieces are pinned
against their definitions (DGESVD pseudo-inverse against numpy's, the
UPDATE_LAMBDA branches, the hat basis), and a short oracle inversion of
synthetic observations must recover the atmosphere it was generated from.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import lm_oracle as lmo  # noqa: E402
import lmcase  # noqa: E402


def test_pinv_matches_numpy_with_cut():
    rng = np.random.default_rng(3)
    for cond in (1e2, 1e6):
        q, _ = np.linalg.qr(rng.standard_normal((13, 13)))
        s = np.logspace(0, -np.log10(cond), 13)
        m = (q * s) @ q.T
        a = lmo.pinv_dgesvd(m, 1e-4)
        b = np.linalg.pinv(m, rcond=1e-4, hermitian=True)
        assert np.allclose(a, b, rtol=1e-9, atol=1e-9 * np.abs(b).max())


def test_update_lambda_branches():
    # big improvement: steps decrease (not below 0), lambda / sqrt(10)
    assert lmo.update_lambda(1.0, 2.0, 10.0, 0.0, 0.0) == (1.0, 10.0 / np.sqrt(10.0), 0.0, 0.0)
    # small improvement (< 1 %): steps increase
    c, lam, st, pc = lmo.update_lambda(0.999, 1.0, 1.0, 2.0, 0.0)
    assert (c, st) == (0.999, 3.0) and np.isclose(lam, 1.0 / np.sqrt(10.0))
    # no improvement: lambda x 10; after a PRECYC = 1 cycle: x 3 and PRECYC reset
    assert lmo.update_lambda(2.0, 1.0, 1.0, 0.0, 0.0) == (1.0, 10.0, 1.0, 0.0)
    assert lmo.update_lambda(2.0, 1.0, 1.0, 0.0, 1.0) == (1.0, 3.0, 1.0, 0.0)
    # floor 1e-2
    assert lmo.update_lambda(0.5, 1.0, 0.01, 0.0, 0.0)[1] == 0.01


def test_hat_basis_partition_of_unity():
    for nz, nj in ((48, 5), (128, 2), (128, 13), (64, 64)):
        c = lmo.int_coefs(nz, nj)
        assert np.allclose(c.sum(axis=1), 1.0)
        assert c.shape == (nz, nj)


def test_oracle_inversion_recovers_the_atmosphere(fz, orc):
    lines = orc.parse_lines(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    nz = 48
    true = fz.atmos.make_columns(3, nz, seed=12)
    obs, true_he, _ = orc.forward(lines, reg, g, true, hydrostatic=True)
    obs = obs.reshape(3, -1)
    init = lmcase.initial_guess(true_he, seed=1)
    w = lmo.weights(obs.shape[1] // 4, isigma=1e-3)
    f = lmcase.oracle_forward_rf(orc, lines, reg, g, he=True)
    syn0, _, _, _ = f(init)
    chi0 = np.sum((obs - syn0) ** 2 * w, axis=1) / obs.shape[1]
    best, chi, it = lmo.invert(f, obs, init, lmcase.NODES, w, maxsteps=5, maxit=25)
    # The reference's step keeps every node direction whose singular value is
    # above 1e-4 of the largest (RSVDTOL) and re-projects the model on the
    # node basis at every step (NODE_EXPANSION = 1); with T dominating H
    # through the hydrostatic coupling it stops well before the noise level,
    # by the STEPS > MAXSTEPS rule.
    assert np.all(chi < 0.2 * chi0), (chi0, chi)
    assert np.all(it < 25)
    assert np.all(np.isfinite(best))


def test_it_penalties_operators():
    """GET_IT_PENALTIES: type 0 is diag(1/NJ), type 1 first differences to the
    previous node, both scaled by sqrt(PEN_ALP / IFREEP); PEN_RES = PEN_HSS x
    with x the node averages over PARAM_NORM; parameters with zero alpha add
    nothing."""
    nz = 40
    nodes = {1: 4, 4: 2, 6: 3}
    rng = np.random.default_rng(2)
    model = np.zeros((13, nz), dtype=np.float32)
    model[0] = 6000.0 + 200.0 * rng.standard_normal(nz)
    model[5] = 300.0 * rng.standard_normal(nz)
    model[7] = 500.0 + 100.0 * rng.standard_normal(nz)
    typ = [1, 0, 0, 0, 0, 1, 0, 0]
    alp = [2.0, 0.0, 0.0, 0.5, 0.0, 3.0, 0.0, 0.0]
    res, hss = lmo.it_penalties(model, nodes, typ, alp)
    npar = 9
    assert res.shape == (npar,) and hss.shape == (npar, npar)
    x = np.concatenate([lmo.contract(model[lmo.ATMPOS[p]], lmo.int_coefs(nz, n)) / lmo.PARAM_NORMS[p - 1]
                        for p, n in sorted(nodes.items())])
    np.testing.assert_allclose(res, hss @ x, rtol=1e-12, atol=1e-15)
    d = np.zeros((4, 4))
    for k in range(1, 4):
        d[k, k], d[k, k - 1] = 1.0, -1.0
    np.testing.assert_allclose(hss[:4, :4], 2.0 / npar * d.T @ d, rtol=1e-12)
    np.testing.assert_allclose(hss[4:6, 4:6], 0.5 / npar * np.eye(2) / 4.0, rtol=1e-12)
    d3 = np.zeros((3, 3))
    for k in range(1, 3):
        d3[k, k], d3[k, k - 1] = 1.0, -1.0
    np.testing.assert_allclose(hss[6:, 6:], 3.0 / npar * d3.T @ d3, rtol=1e-12)
    assert np.all(hss[:4, 4:] == 0) and np.all(hss[4:6, 6:] == 0)
    res0, hss0 = lmo.it_penalties(model, nodes, typ, [0.0] * 8)
    assert np.all(res0 == 0) and np.all(hss0 == 0)


def test_errors_1d_analytic():
    """GET_ERROR_1D with one T node and a Jacobian of known normalised
    Gram diagonal: sigma = sqrt((chi2/INU) / H_11), the height profile is
    that constant times PARAM_NORM (one node expands to a flat profile),
    clipped at 0.15 PARAM_NORM; every other row is zero."""
    nf, nz = 8, 6
    w = np.full(nf, 4.0)
    obs = np.zeros(nf)
    syn = np.full(nf, 0.5)                     # chi2 = sum(0.25 * 4) / 8 = 1
    for scale, expect in ((1.0e-3, None), (1.0e-6, 0.15 * 6000.0)):
        jac = np.full((nf, 1), scale, dtype=np.float32)
        model = np.zeros((13, nz), dtype=np.float32)
        err, chi = lmo.errors_1d(obs, syn, jac, model, w, {1: 1})
        assert chi == pytest.approx(1.0)
        jn = np.float64(np.float32(scale)) * np.sqrt(4.0) / np.sqrt(nf) * 6000.0
        sigma = np.sqrt((1.0 / nf) / (nf * jn * jn)) * 6000.0
        want = min(sigma, 0.15 * 6000.0) if expect is None else expect
        np.testing.assert_allclose(err[0], want, rtol=1e-6)
        assert np.all(err[1:] == 0)


def test_cg_delta_and_node_expansion_two():
    """The oracle's NEW_CALCULATE_DELTA_UBICGSTAB meets its own stopping test
    and tends to the exact solution on an SPD system; SORT_DELTA with
    NODE_EXPANSION = 2 makes the new profile the expansion of the node values
    plus the clipped node deltas (limits aside)."""
    rng = np.random.default_rng(3)
    m = rng.standard_normal((13, 13))
    a = m @ m.T + 13 * np.eye(13)
    b = rng.standard_normal(13)
    x = lmo.cg_delta(a, b)
    assert np.sum(((a @ x - b) / (np.abs(b) + 1e-5)) ** 2) / 13 < 1e-3
    np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=0.1, atol=1e-3)
    nz, nj = 40, 5
    coefs = lmo.int_coefs(nz, nj)
    ipar = np.linspace(9000.0, 4500.0, nz).astype(np.float32)
    delta = np.array([0.01, -0.02, 0.0, 0.015, -0.01])
    pert2, itd = lmo.sort_delta(delta, 6000.0, ipar, 2500.0, 1.8e4, coefs, 900.0, node_expansion=2)
    avg = lmo.contract(ipar, coefs)
    want = (lmo.expand(avg + itd, coefs).astype(np.float32) - ipar).astype(np.float32)
    np.testing.assert_array_equal(pert2, want)


def test_record_is_the_state_of_the_stopped_inversion(fz, orc):
    """The per-iteration record of the oracle's inversion (what the GPU is
    compared with, iteration by iteration) equals the final state of the
    same inversion stopped at maxit = k."""
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2, nw=24), lines)
    g, _ = orc.gain(lines, reg)
    nz, npix = 32, 4
    true = fz.atmos.make_columns(npix, nz, seed=71)
    obs, _, _ = orc.forward(lines, reg, g, true, hydrostatic=False)
    obs = obs.reshape(npix, -1) + np.random.default_rng(1).normal(0.0, 1e-3, (npix, obs.shape[1] * obs.shape[2]))
    init = lmcase.initial_guess(true, seed=1)
    w = lmo.weights(obs.shape[1] // 4, isigma=1e-3)
    f = lmcase.oracle_forward_rf(orc, lines, reg, g, False)
    rec = []
    lmo.invert(f, obs, init, lmcase.NODES, w, maxit=3, record=rec)
    assert len(rec) == 3
    for k in (1, 2, 3):
        best, chi, it = lmo.invert(f, obs, init, lmcase.NODES, w, maxit=k)
        assert np.all(it == k)
        for i in range(npix):
            assert rec[k - 1][i][2] == chi[i]
            assert np.array_equal(rec[k - 1][i][5], best[i])
