"""GPU response functions against the FP64 oracle.

The GPU evaluates the response functions in FP32 (the library's precision
split: FP64 only for the chemistry, the pressure integration and the LM
solve) and accumulates the node Jacobian forward along z; the oracle restates
the reference's FP64 chain (local RFs, OLD_DSYN_PROPAGATION,
CALCULATE_EQUIVALENT_DSYN).  Each Jacobian column (one node of one parameter,
all Stokes parameters and wavelengths) is compared relative to its own
largest entry:

    max |J_gpu - J_oracle| <= RF_TOL * max |J_oracle|     (RF_TOL = 2e-4)

(FP32 against FP64 measures ~3e-5; the bound leaves a 6x margin and still
catches a wrong term in any one parameter's derivative chain)

and the Stokes vector of the same call to the synthesis tolerances (1e-5
relative in I, 1e-6 absolute in Q, U, V).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RF_TOL = 2e-4


def _setup(fz, orc, nz, ncol, seed):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    m = fz.atmos.make_columns(ncol, nz, seed=seed)
    return lines, reg, g, m


def _compare(fz, orc, lines, reg, g, m, nodes, he):
    nz = m.shape[2]
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    np_ = ctx.rf_nodes(nodes)
    syn, jac, mo, st = ctx.forward_rf(m, hydrostatic=he)
    osyn, ojac, omo, ost = orc.forward_rf(lines, reg, g, m, nodes, hydrostatic=he)
    assert np.all(st == 0) and np.all(ost == 0)
    assert jac.shape == ojac.shape == (m.shape[0], np_, 4 * syn.shape[2])
    assert np.max(np.abs(syn[:, 0] - osyn[:, 0]) / np.abs(osyn[:, 0])) < 1e-5
    assert np.max(np.abs(syn[:, 1:] - osyn[:, 1:])) < 1e-6
    scale = np.abs(ojac).max(axis=2)                          # (ncol, np)
    err = np.abs(jac.astype(np.float64) - ojac).max(axis=2)
    rel = err / np.where(scale > 0, scale, 1.0)
    return rel, scale


@pytest.mark.parametrize("he", [True, False])
def test_node_jacobian_matches_oracle(fz, orc, he):
    lines, reg, g, m = _setup(fz, orc, nz=64, ncol=8, seed=31)
    if not he:
        _, m, _ = orc.forward(lines, reg, g, m, hydrostatic=True)
        nodes = {1: 5, 2: 3, 4: 2, 5: 2, 6: 2, 7: 2}
    else:
        nodes = {1: 5, 4: 2, 5: 2, 6: 2, 7: 2}   # the inversion's node layout
    rel, scale = _compare(fz, orc, lines, reg, g, m, nodes, he)
    assert np.all(scale > 0)
    assert rel.max() <= RF_TOL, rel.max()


@pytest.mark.parametrize("p", [1, 2, 6, 7])
def test_height_response_functions_match_oracle(fz, orc, p):
    lines, reg, g, m = _setup(fz, orc, nz=48, ncol=4, seed=7)
    _, m, _ = orc.forward(lines, reg, g, m, hydrostatic=True)
    rel, scale = _compare(fz, orc, lines, reg, g, m, {p: 48}, he=False)
    # heights whose response is negligible (deep, optically thick) are
    # compared against the strongest height of the same column instead
    colmax = scale.max(axis=1, keepdims=True)
    rel = rel * scale / colmax
    assert rel.max() <= RF_TOL, rel.max()


def test_rf_nodes_validation(fz, orc):
    lines, reg, g, m = _setup(fz, orc, nz=32, ncol=1, seed=1)
    ctx = fz.Synthesis(lines, reg, nz=32, gain=g)
    with pytest.raises(fz.FzError):
        ctx.rf_nodes({3: 2})            # rho is not a response-function parameter here
    with pytest.raises(fz.FzError):
        ctx.rf_nodes({1: 33})           # more nodes than heights
    with pytest.raises(fz.FzError):
        ctx.forward_rf(m)               # no node layout yet


@pytest.mark.parametrize("he", [True, False])
@pytest.mark.parametrize("nz,ncol", [(32, 4), (128, 2)])
def test_full_height_rf_matches_oracle(fz, orc, he, nz, ncol):
    """fz_forward_rf_full: the WRITE RESPONSE FUNCTION output (one node per
    height for T, Pg, Bx, By, Bz, v_z) against the oracle's EQVDSYN with
    NJ = NZ, at 32 heights and at the benchmark's 128; heights compared
    against the strongest height of the same (column, parameter)."""
    lines, reg, g, m = _setup(fz, orc, nz=nz, ncol=ncol, seed=11)
    if not he:
        _, m, _ = orc.forward(lines, reg, g, m, hydrostatic=True)
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    syn, rf, mo, st = ctx.forward_rf_full(m, hydrostatic=he)
    nodes = {1: nz, 2: nz, 4: nz, 5: nz, 6: nz, 7: nz}
    osyn, ojac, _, ost = orc.forward_rf(lines, reg, g, m, nodes, hydrostatic=he)
    assert np.all(st == 0) and np.all(ost == 0)
    assert rf.shape == (m.shape[0], 6, nz, 4 * syn.shape[2])
    assert np.max(np.abs(syn[:, 0] - osyn[:, 0]) / np.abs(osyn[:, 0])) < 1e-5
    assert np.max(np.abs(syn[:, 1:] - osyn[:, 1:])) < 1e-6
    o = ojac.reshape(rf.shape)
    err = np.abs(rf.astype(np.float64) - o).max(axis=3)           # (ncol, 6, nz)
    pmax = np.abs(o).max(axis=(2, 3))                               # (ncol, 6)
    assert np.all(pmax > 0)
    rel = err / pmax[:, :, None]
    assert rel.max() <= RF_TOL, rel.max()


@pytest.mark.parametrize("he", [True, False])
def test_full_height_rf_contracts_to_node_jacobian(fz, orc, he):
    """At the benchmark's height grid: the hat-function contraction of the
    response functions at every height equals the node Jacobian of the node
    path (CALCULATE_EQUIVALENT_DSYN is linear in DSYN1D), to FP32 rounding."""
    from firtez_dz_b200 import warmstart as ws
    nz = 128
    lines, reg, g, m = _setup(fz, orc, nz=nz, ncol=16, seed=5)
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    nodes = {1: 5, 2: 3, 4: 2, 5: 2, 6: 2, 7: 2}
    ctx.rf_nodes(nodes)
    _, jac, _, st1 = ctx.forward_rf(m, hydrostatic=he)
    _, rf, _, st2 = ctx.forward_rf_full(m, hydrostatic=he)
    assert np.all(st1 == 0) and np.all(st2 == 0)
    cols = []
    for slot, p in enumerate((1, 2, 4, 5, 6, 7)):
        c = ws.hat_coefs(nz, nodes[p])                               # (nz, nj)
        cols.append(np.einsum("kj,nkf->njf", c, rf[:, slot].astype(np.float64)))
    jc = np.concatenate(cols, axis=1)
    scale = np.abs(jac).max(axis=2, keepdims=True)
    assert np.all(scale > 0)
    assert np.max(np.abs(jc - jac) / scale) <= 1e-4
