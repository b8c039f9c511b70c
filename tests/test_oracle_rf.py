"""Pins of the response-function half of the FP64 oracle.

The reference has no golden response functions (its test_rf case writes them
without expected values), so the oracle's RFs are pinned the way the
reference itself checks them (src/invert3d.f90:93-138): against central
finite differences of the synthesis, plus the identities the reference's
formulas imply where they are deliberately not the exact derivative:

* hydrostatic T: RF_T = RF_T|Pg + sum_{I<K} RF_Pg(I) * DPGDTK_HE(I)
  (src/forward.f90:1050-1057, src/rtesolver.f90:218-232);
* hydrostatic B and v_z: the reference evaluates them with the layer's
  outgoing Stokes vector (STKIN is reassigned at src/rtesolver.f90:230), so
  they differ from finite differences in deep layers; this is restated on
  purpose and only the non-hydrostatic B/v RFs are compared with finite
  differences.
"""
import numpy as np
import pytest

MAMU = 1.66053892e-24
KBOL = 1.38056503e-16
GRAV = 2.7414e4
NZ = 48


@pytest.fixture(scope="module")
def setup(fz, orc):
    lines = orc.parse_lines(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    m = fz.atmos.make_columns(2, NZ, seed=5)
    _, m_he, _ = orc.forward(lines, reg, g, m, hydrostatic=True)
    return lines, reg, g, m, m_he


def test_rf_path_keeps_stokes_bit_exact(setup, orc):
    lines, reg, g, m, m_he = setup
    for he, mod in ((True, m), (False, m_he)):
        st, jac, mo, s = orc.forward_rf(lines, reg, g, mod, {1: 5, 4: 2, 5: 2, 6: 2, 7: 2}, hydrostatic=he)
        st0, mo0, s0 = orc.forward(lines, reg, g, mod, hydrostatic=he)
        assert np.array_equal(st, st0) and np.array_equal(mo, mo0)
        assert np.all(s == 0) and np.all(np.isfinite(jac))
        assert jac.shape == (2, 13, 4 * st.shape[2])


ROWS = {1: 0, 2: 1, 4: 5, 5: 6, 6: 7, 7: 10}


@pytest.mark.parametrize("p", [1, 2, 4, 5, 6, 7])
def test_nonhydrostatic_rf_matches_finite_differences(setup, orc, p):
    lines, reg, g, _, m = setup
    nodes = {q: NZ for q in (1, 2, 4, 5, 6, 7)}
    _, jac, _, _ = orc.forward_rf(lines, reg, g, m[:1], nodes, hydrostatic=False)
    order = [1, 2, 4, 5, 6, 7]
    for k in (12, 20, 28):
        step = {1: 1.0, 2: float(m[0, 1, k]) * 1e-4, 4: 1.0, 5: 1.0, 6: 1.0, 7: 100.0}[p]
        mp, mm = m[:1].copy(), m[:1].copy()
        mp[0, ROWS[p], k] += step
        mm[0, ROWS[p], k] -= step
        h = float(mp[0, ROWS[p], k] - mm[0, ROWS[p], k]) / 2.0
        sp, _, _ = orc.forward(lines, reg, g, mp, hydrostatic=False)
        sm, _, _ = orc.forward(lines, reg, g, mm, hydrostatic=False)
        fd = ((sp - sm) / (2.0 * h))[0].reshape(-1)
        an = jac[0, order.index(p) * NZ + k].astype(np.float64)
        scale = np.abs(fd).max()
        # T goes through GET_RHO's 1e-4 fixed point in the finite difference
        tol = 2e-3 if p == 1 else 3e-4
        assert np.abs(fd - an).max() <= tol * scale, (p, k)


def test_hydrostatic_temperature_rf_identity(setup, orc):
    lines, reg, g, m, _ = setup
    _, jhe, mo, _ = orc.forward_rf(lines, reg, g, m[:1], {1: NZ}, hydrostatic=True)
    _, jn, _, _ = orc.forward_rf(lines, reg, g, mo, {1: NZ, 2: NZ}, hydrostatic=False)
    T, PG, MW = mo[0, 0], mo[0, 1], mo[0, 4]
    Z = mo[0, 12].astype(np.float64)
    jT, jP = jn[0, :NZ].astype(np.float64), jn[0, NZ:].astype(np.float64)
    pred = jT.copy()
    for K in range(1, NZ):
        cte = MAMU / KBOL * GRAV * (Z[K] - Z[K - 1]) * 1e3 * 1e2
        h = -(float(np.float32(PG[K] * MW[K])) * cte / float(T[K]) / float(T[K]))
        for I in range(K):
            pred[K] += float(np.float32(PG[I] / PG[K])) * h * jP[I]
    got = jhe[0].astype(np.float64)
    for K in range(10, NZ):
        scale = np.abs(got[K]).max()
        # HE and non-HE runs differ in the electron density they feed the
        # opacities (initial-guess Pe vs converged ne), ~1e-5 relative
        assert np.abs(got[K] - pred[K]).max() <= 2e-4 * scale, K
    # the global term matters: without it the upper layers are wrong
    assert np.abs(got[40] - jT[40]).max() > 0.5 * np.abs(got[40]).max()


def test_node_jacobian_is_hat_contraction_of_height_rf(setup, orc):
    lines, reg, g, _, m = setup
    _, jfull, _, _ = orc.forward_rf(lines, reg, g, m[:1], {1: NZ, 7: NZ}, hydrostatic=False)
    _, jnod, _, _ = orc.forward_rf(lines, reg, g, m[:1], {1: 5, 7: 2}, hydrostatic=False)
    for p, nj, off_f, off_n in ((1, 5, 0, 0), (7, 2, NZ, 5)):
        step = (NZ - 1) / (nj - 1)
        pos = np.arange(nj) * step                    # 0-based node heights
        z = np.arange(NZ, dtype=np.float64)
        for j in range(nj):
            c = np.clip(1.0 - np.abs(z - pos[j]) / step, 0.0, None)
            pred = c @ jfull[0, off_f:off_f + NZ].astype(np.float64)
            got = jnod[0, off_n + j].astype(np.float64)
            assert np.abs(got - pred).max() <= 1e-5 * np.abs(pred).max(), (p, j)


def test_rf_rejects_unsupported_parameters(setup, orc):
    lines, reg, g, _, m = setup
    with pytest.raises(ValueError):
        orc.forward_rf(lines, reg, g, m[:1], {3: 2}, hydrostatic=False)
    with pytest.raises(ValueError):
        orc.forward_rf(lines, reg, g, m[:1], {1: NZ + 1}, hydrostatic=False)
