"""Pins of the oracle that do not go through its own restatement.

The reference has no golden Stokes outputs and cannot be built here, so the
oracle's Voigt function and formal solution are checked against independent
mathematics:

* VOIGT (src/voigt.f:17-98) is Hui, Armstrong & Wray's rational
  approximation of the Faddeeva function: H(a, v) = Re w(v + i a) and
  F(a, v) = Im w(v + i a) (the reference's FF carries the factor 2 that
  makes it Im w).  Against scipy.special.wofz the 7-pole form is accurate to
  5e-6 absolute for damping a >= 1e-4 over |v| <= 25 (its published accuracy
  class; the error peaks at the knee between core and wings).
* The evolution-operator formal solution (EVOL_OPERATOR + OLD_ANALYTICAL_
  SOLVER, src/rtesolver.f90:163-473) is exact for a source function that is
  constant within each layer: I_K = (1 - O_K) S_K e0 + O_K I_{K-1} with
  O_K = exp(-K_K dz_K), K the 4x4 absorption matrix
  [[eI, eQ, eU, eV], [eQ, eI, -rV, rU], [eU, rV, eI, -rQ], [eV, -rU, rQ, eI]].
  The oracle's closed form (Landi Degl'Innocenti's M2, M3, M4 algebra) is
  compared with the same recursion built on scipy.linalg.expm (Pade).
* Unno-Rachkovsky: for a Milne-Eddington slab (K / kappa_c constant, S = S0 +
  S1 tau_c) the emergent Stokes vector is S0 e0 + S1 (K / kappa_c)^-1 e0; the
  recursion approaches it as the layers thin -- at second order in dtau with
  each layer's source taken at its optical-depth midpoint, at first order
  with the value at its top.
"""
import numpy as np
import pytest
from scipy.linalg import expm
from scipy.special import wofz


def absorption_matrix(ei, eq, eu, ev, rq, ru, rv):
    return np.array([[ei, eq, eu, ev], [eq, ei, -rv, ru], [eu, rv, ei, -rq], [ev, -ru, rq, ei]])


def zeeman_like_eta(rng, nw, scale):
    """Seven absorption-matrix rows (7, nw) of a physical matrix: eta_I >
    |(eta_Q, eta_U, eta_V)|, magneto-optical terms of the same order."""
    line = rng.uniform(0.0, 20.0, nw)
    d = rng.normal(0.0, 1.0, (3, nw))
    d /= np.linalg.norm(d, axis=0)
    pol = line * rng.uniform(0.0, 0.9, nw)
    eta = np.zeros((7, nw))
    eta[0] = 1.0 + line
    eta[1:4] = d * pol
    eta[4:7] = rng.normal(0.0, 0.5, (3, nw)) * line
    return eta * scale


def expm_solution(eta, src, zz, bnd=None):
    """The recursion of OLD_ANALYTICAL_SOLVER with O = expm(-K dz)."""
    nz, _, nw = eta.shape
    out = np.zeros((nw, 4))
    for k in range(nz):
        if k == 0 or (bnd is not None and bnd[k]):
            out[:, 0] = src[k]
            out[:, 1:] = 0.0
            continue
        dz = 1e5 * abs(zz[k] - zz[k - 1]) if k == nz - 1 else 1e5 * abs(zz[k + 1] - zz[k])
        for lam in range(nw):
            O = expm(-absorption_matrix(*eta[k, :, lam]) * dz)
            e0 = np.array([1.0, 0.0, 0.0, 0.0])
            out[lam] = (e0 - O[:, 0]) * src[k, lam] + O @ out[lam]
    return out


def me_slab(nz, tau_max, rng, nw=6, kc=1e-7):
    """A Milne-Eddington slab on a log grid in continuum optical depth: one
    matrix K / kappa_c for all heights, heights z (km) from tau_c."""
    kt = zeeman_like_eta(rng, nw, 1.0)                      # K / kappa_c
    # bottom -> top; the top height's layer (the backward difference of the
    # reference's dz rule counts it twice) is made optically negligible
    tau = np.concatenate([np.geomspace(tau_max, 1e-9, nz - 1), [0.0]])
    # tau_c at height K counts the layers above it: dz_K = (tau_K - tau_{K+1}) / kappa_c
    zz = np.zeros(nz)
    for k in range(nz - 2, -1, -1):
        zz[k] = zz[k + 1] - (tau[k] - tau[k + 1]) / kc / 1e5
    eta = np.repeat((kt * kc)[None], nz, axis=0)
    return eta, tau, zz, kt


@pytest.mark.parametrize("a", [1e-4, 1e-3, 1e-2, 0.1, 0.5, 1.0, 3.0])
def test_voigt_is_the_faddeeva_function(orc, a):
    v = np.linspace(-25.0, 25.0, 4001)
    h, f = orc.voigt(a, v)
    w = wofz(v + 1j * a)
    assert np.max(np.abs(h - w.real)) < 5e-6, a
    assert np.max(np.abs(f - w.imag)) < 5e-6, a
    # the normalisation of the header comment: the integral of H is sqrt(pi)
    if a >= 0.1:
        vv = np.linspace(-2000.0, 2000.0, 800001)
        hh, _ = orc.voigt(a, vv)
        integ = np.trapezoid(hh, vv) + 2.0 * a / (np.sqrt(np.pi) * 2000.0)   # + the far wings, H ~ a / (sqrt(pi) v^2)
        assert abs(integ / np.sqrt(np.pi) - 1.0) < 2e-4, a


def test_formal_solution_is_the_matrix_exponential_recursion(orc):
    """Random physical matrices per height, a source function per height and
    wavelength, a boundary flag inside the slab: the oracle's closed-form
    operators reproduce the expm recursion to rounding."""
    rng = np.random.default_rng(7)
    nz, nw = 24, 5
    eta = np.stack([zeeman_like_eta(rng, nw, 1e-7) for _ in range(nz)])
    zz = np.cumsum(rng.uniform(5.0, 40.0, nz))                  # km, ascending: dtau ~ 0.05-0.4 per layer
    src = rng.uniform(0.5, 2.0, (nz, nw))
    bnd = np.zeros(nz, dtype=np.int32)
    bnd[6] = 1
    for b in (None, bnd):
        got = orc.rte_solve(eta, src, zz, b)
        ref = expm_solution(eta, src, zz, b)
        assert np.max(np.abs(got - ref)) < 1e-12 * np.max(np.abs(ref)), b is None


def test_unno_rachkovsky_limit(orc):
    """Milne-Eddington slab: the recursion tends to the Unno-Rachkovsky
    solution S0 e0 + S1 (K/kappa_c)^-1 e0, the error falling 4x per halving
    of the layers with midpoint sources (to 3.5e-6 at 4000 layers) and 2x
    with top-of-layer sources."""
    s0, s1 = 0.4, 1.3
    err = {}
    for nz in (2001, 4001):
        eta, tau, zz, kt = me_slab(nz, 40.0, np.random.default_rng(3))
        tnext = np.concatenate([tau[1:], [0.0]])
        ur = np.stack([s0 * np.eye(4)[0] + s1 * np.linalg.solve(absorption_matrix(*kt[:, lam]), np.eye(4)[0])
                       for lam in range(kt.shape[1])])
        for name, t in (("mid", 0.5 * (tau + tnext)), ("top", tnext)):
            src = np.repeat((s0 + s1 * t)[:, None], eta.shape[2], axis=1)
            err[(name, nz)] = np.max(np.abs(orc.rte_solve(eta, src, zz) - ur))
    assert err[("mid", 4001)] < 5e-6 * s1, err
    assert 3.6 < err[("mid", 2001)] / err[("mid", 4001)] < 4.4, err
    assert 1.8 < err[("top", 2001)] / err[("top", 4001)] < 2.2, err
