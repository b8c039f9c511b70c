"""TEST INFRASTRUCTURE -- not part of the product.

numpy restatement of SET_TAU's assists (src/invert3d.f90:492-727), the
checker of fz_set_tau(_device).  obs (NX*NY, 4, NUMW) REAL*8 with pixel
iy + NY ix (OBS3D(NFREQ,NY,NX)); models (NX*NY, 13, NZ) REAL*4; n1 = NUMWAVE
of the first spectral region; l0 = LINE_L0(IND_LINE(1)) [A].

  VECTORS(:,1) = SUM(SUM(OBS3D(region 1 of I,:,:),DIM=2),DIM=2) / SUM(ABS(.))
  VECTORS(:,2..3) = centred derivatives, ends copied, / SUM(ABS(.))
  B   TAU(3) = V.v2 / MAXVAL|.|, TAU(4) = |(Q.v3, U.v3)| / MAXVAL,
      ATN2 = ATAN2(U.v3, Q.v3)/2, Bx = -REAL(SIN(ATN2))*1000*TAU(4),
      By = REAL(COS(ATN2))*1000*TAU(4), Bz = REAL(TAU(3))*(-1000)    :519-571
  V   D = I.v2 - (I.v1) KOL, KOL = v2.v1, vz = REAL(D/MAXVAL|D|)*(-2e5) :572-628
  T   Tb = 1/(LK_HC ln(1 + (exp(1/6390/LK_HC) - 1)/mean I)), T += Tb - T(ITZ) :630-655
  P   Pg = Pg*1.333e5/Pg(ITZ) (REAL*4)                                   :656-672
  ITZ = CEILING(REAL(NZ)/3); with T or P log tau5 = 1 except 0 at ITZ, then
  the plain synthesis (HYDRO_TOP off) rewrites rho, Pe, mu, log tau5 -- left
  to the caller (the library's and the oracle's forward solvers).
"""
import numpy as np

KBOL = 1.38056503e-16
HPLA = 6.62606957e-27
LIGHT = 2.99792458e10


def vectors(obs, nx, ny, n1):
    i1 = obs[:, 0, :n1].reshape(nx, ny, n1)
    tot = np.zeros(n1)
    for ix in range(nx):            # the y sum of each x first, then over x
        t = np.zeros(n1)
        for iy in range(ny):
            t = t + i1[ix, iy]
        tot = tot + t

    def deriv(a):
        b = np.empty_like(a)
        b[1:-1] = (a[2:] - a[:-2]) / 2.0
        b[0], b[-1] = b[1], b[-2]
        return b

    v1 = tot / np.sum(np.abs(tot))
    v2 = deriv(v1)
    v2 = v2 / np.sum(np.abs(v2))
    v3 = deriv(v2)
    v3 = v3 / np.sum(np.abs(v3))
    return v1, v2, v3


def set_tau(obs, models, nx, ny, n1, l0, assist):
    """assist: set of 'temp', 'pgas', 'bvec', 'vlos'.  Returns new models
    (before the forward synthesis of the T/P assists)."""
    m = np.array(models, dtype=np.float32, copy=True)
    nz = m.shape[2]
    v1, v2, v3 = vectors(obs, nx, ny, n1)
    kol = float(np.dot(v2, v1))
    I, Q, U, V = (obs[:, s, :n1] for s in range(4))
    if "bvec" in assist:
        t3 = V @ v2
        tq, tu = Q @ v3, U @ v3
        t3 = t3 / np.max(np.abs(t3))
        t4 = np.sqrt(tq ** 2 + tu ** 2)
        t4 = t4 / np.max(t4)
        atn2 = np.arctan2(tu, tq) / 2.0
        bx = ((-np.sin(atn2).astype(np.float32) * np.float32(1000.0)).astype(np.float64) * t4).astype(np.float32)
        by = ((np.cos(atn2).astype(np.float32) * np.float32(1000.0)).astype(np.float64) * t4).astype(np.float32)
        bz = t3.astype(np.float32) * np.float32(-1000.0)
        m[:, 5, :], m[:, 6, :], m[:, 7, :] = bx[:, None], by[:, None], bz[:, None]
    if "vlos" in assist:
        d = I @ v2 - (I @ v1) * kol
        d = d / np.max(np.abs(d))
        m[:, 10, :] = (d.astype(np.float32) * np.float32(-2.0e5))[:, None]
    itz = int(np.ceil(np.float32(nz) / np.float32(3.0))) - 1
    if "temp" in assist:
        imean = np.sum(I, axis=1) / float(n1)
        lk = (l0 * 1.0e-8 * KBOL) / (HPLA * LIGHT)
        tb = 1.0 / (lk * np.log(1.0 + 1.0 / imean * (np.exp(1.0 / 6.39e3 / lk) - 1.0)))
        sh = tb - m[:, 0, itz].astype(np.float64)
        m[:, 0, :] = (m[:, 0, :].astype(np.float64) + sh[:, None]).astype(np.float32)
    if "pgas" in assist:
        p0 = m[:, 1, itz].copy()
        m[:, 1, :] = m[:, 1, :] * np.float32(1.333e5) / p0[:, None]
    if "temp" in assist or "pgas" in assist:
        m[:, 11, :] = np.float32(1.0)
        m[:, 11, itz] = np.float32(0.0)
    return m
