"""Seeded synthetic model atmospheres and the line sets of the benchmark workloads.

There is no public dataset for this path; these generators stand in for the
reference's MHD/inverted cubes with the shapes and distributions below.

Column model (MODEL(NZ,13) REAL*4, index 0 = bottom):
  * z uniform from -500 to +1500 km;
  * T(z): monotone radiative-equilibrium-like profile from 9500 K (bottom) to
    4300 K (top) plus a Gaussian random field, sigma 150 K, correlation length
    100 km (covariance exp(-dz^2 / (2 l^2)));
  * Pg: hydrostatic, d ln Pg / dz = -mu m_u g / (k T) with mu = 1.3, from
    Pg(z = 0) = 1.2e5 dyn cm^-2 (the synthesis recomputes rho, Pe, mu by
    chemical equilibrium, or re-integrates Pg from the top in hydrostatic mode);
  * |B| ~ U(0, bmax) G, cos(gamma) ~ U(-1, 1), phi ~ U(0, pi),
    v_z ~ N(0, 2 km/s) in cm/s; each constant per column times a 10 % linear
    decrease from bottom to top;
  * rho, Pe, mu, log tau5, vx, vy = 0.
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
KBOL = 1.38056503e-16
MAMU = 1.66053892e-24
GRAV = 2.7414e4


def z_grid(nz, zmin=-500.0, zmax=1500.0):
    return np.linspace(zmin, zmax, nz)


def mean_temperature(z, tbot=9500.0, ttop=4300.0, h=552.0):
    s = z - z[0]
    span = z[-1] - z[0]
    etop = np.exp(-span / h)
    f = (np.exp(-s / h) - etop * s / span) / (1.0 - etop)
    return ttop + (tbot - ttop) * f


def correlated_noise(rng, n, z, sigma, corr):
    """Gaussian random field on grid z with covariance sigma^2 exp(-dz^2/(2 corr^2))."""
    dz = z[:, None] - z[None, :]
    cov = sigma ** 2 * np.exp(-0.5 * (dz / corr) ** 2) + 1e-9 * sigma ** 2 * np.eye(len(z))
    L = np.linalg.cholesky(cov)
    return rng.standard_normal((n, len(z))) @ L.T


def hydrostatic_pg(T, z, pg0=1.2e5, z0=0.0, mu=1.3):
    """ln Pg integrated with the trapezoid rule from z0 (km) both ways."""
    zc = z * 1e5
    g = -mu * MAMU * GRAV / (KBOL * T)           # d ln P / dz  [1/cm], (ncol, nz)
    seg = 0.5 * (g[:, 1:] + g[:, :-1]) * np.diff(zc)[None, :]
    lnp = np.concatenate([np.zeros((T.shape[0], 1)), np.cumsum(seg, axis=1)], axis=1)
    # anchor at z0 by linear interpolation of ln P
    k = int(np.clip(np.searchsorted(z, z0) - 1, 0, len(z) - 2))
    w = (z0 - z[k]) / (z[k + 1] - z[k])
    ref = (1 - w) * lnp[:, k] + w * lnp[:, k + 1]
    return pg0 * np.exp(lnp - ref[:, None])


def make_columns(ncol, nz, seed, bmax=2500.0, tsig=150.0, corr=100.0):
    """(ncol, 13, nz) float32 columns (C order == Fortran MODEL(NZ,13,ncol))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    z = z_grid(nz)
    T = mean_temperature(z)[None, :] + correlated_noise(rng, ncol, z, tsig, corr)
    T = np.maximum(T, 3000.0)
    pg = hydrostatic_pg(T, z)
    bmod = rng.uniform(0.0, bmax, ncol)
    cosg = rng.uniform(-1.0, 1.0, ncol)
    phi = rng.uniform(0.0, np.pi, ncol)
    vz = rng.normal(0.0, 2.0e5, ncol)
    sing = np.sqrt(np.maximum(0.0, 1.0 - cosg ** 2))
    grad = 1.0 - 0.1 * (z - z[0]) / (z[-1] - z[0])
    m = np.zeros((ncol, 13, nz), dtype=np.float32)
    m[:, 0] = T
    m[:, 1] = pg
    m[:, 5] = (bmod * sing * np.cos(phi))[:, None] * grad
    m[:, 6] = (bmod * sing * np.sin(phi))[:, None] * grad
    m[:, 7] = (bmod * cosg)[:, None] * grad
    m[:, 10] = vz[:, None] * grad
    m[:, 12] = z[None, :]
    return m


def line_database_text():
    with open(os.path.join(HERE, "data", "lines_b200.dat")) as fh:
        return fh.read()


def lines_section(nlines=2, nw=None):
    """LINES: rows of the workloads: Fe I 6301.5 and 6302.5, 112 points of
    21.5 mA centred on each line; with nlines=4 also Fe I 15648.5 and 15652.9
    (96 points each)."""
    if nlines == 2:
        n = nw or 112
        return "1 %d %.2f 21.5\n2 %d %.2f 21.5\n" % (n, -(n - 1) * 21.5 / 2, n, -(n - 1) * 21.5 / 2)
    n = nw or 96
    st = -(n - 1) * 21.5 / 2
    return "1 %d %.2f 21.5\n2 %d %.2f 21.5\n3 %d %.2f 21.5\n4 %d %.2f 21.5\n" % (n, st, n, st, n, st, n, st)
