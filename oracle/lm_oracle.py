"""TEST INFRASTRUCTURE -- not part of the product.

FP64 restatement of FIRTEZ-dz's pixel-wise Levenberg-Marquardt step, used by
tests/ and by the CPU baseline of bench.py as the checker.  The SVD is LAPACK
DGESVD through scipy, the routine the reference itself calls
(src/lm.f90:93-103; LAPACK 3.7/3.9 in the reference's manual).

Followed routines (src/get_dmodel.f90 unless noted):
  GET_PERT_1D :1201-1244, NEW_CALCULATE_CHI2 :960-1032, UPDATE_LAMBDA
  :917-956, NORMALIZE_JACOB :725-770 (PARAM_NORMS :31), NEW_SOLVE_PERTURBATION
  :780-829, GET_PERTURBATION/GET_INVERSE src/lm.f90:61-204, LIMIT_PERTURBATION
  :884-907, REARANGE_DA_MODEL :1843-2016, SORT_DELTA_TO_ATMOSPHERE :1715-1836,
  EXPAND/CONTRACT_VECTOR :839-880, GET_INT_COEFS :563-644, SET_WEIGHTS
  :2024-2047 with the WSTK normalisation of src/input_file.f90:1298-1303,
  INITIALIZE_CYCLE src/invert3d.f90:228-300 (initial state), IFREE_VAR_SPACE
  :411-442 (MPERT = 0.15, RSVDTOL = 1e-4).

Vertical regularisation (GET_IT_PENALTIES), SOLVER_METHOD 1 (SVD) or 2
(conjugate gradients) and NODE_EXPANSION 1 (SIR-like, the reference default,
src/input_file.f90:452-453) or 2 (STiC-like) are options.
"""
import numpy as np
from scipy.linalg import lapack

PARAM_NORMS = np.array([6000.0, 1.0e5, 1.0e-5, 1.0e3, 1.0e3, 1.0e3, 1.0e6, 6.0e2])
LOWLIM = np.array([2500.0, 1.0e-2, 1.0e-10, -5.0e4, -5.0e4, -5.0e4, -1.0e7, 1.0e-8])
UPPLIM = np.array([1.8e4, 1.0e12, 1.0e10, 5.0e4, 5.0e4, 5.0e4, 1.0e7, 1.0e12])
# model row of each reference parameter (src/get_dmodel.f90:1861-1868), 0-based
ATMPOS = {1: 0, 2: 1, 3: 2, 4: 5, 5: 6, 6: 7, 7: 10, 8: 1}
MPERT = 0.15
RSVDTOL = 1.0e-4
TAU_ROW = 11


def int_coefs(nz, nj):
    """GET_INT_COEFS with GET_POSITIONS: (nz, nj) hat coefficients."""
    c = np.zeros((nz, nj))
    if nj == 1:
        c[:, 0] = 1.0
    elif nj < nz:
        step = (nz - 1) / (nj - 1)
        pos = (np.arange(1, nj + 1) - 1.0) * step + 1.0
        for j in range(1, nj + 1):
            ji, jf, jm = pos[max(j - 1, 1) - 1], pos[min(j + 1, nj) - 1], pos[j - 1]
            for i in range(1, nz + 1):
                if i < ji or i > jf:
                    continue
                if i == jm:
                    c[i - 1, j - 1] = 1.0
                elif i < jm:
                    c[i - 1, j - 1] = 1.0 / (jm - ji) * (i - ji)
                else:
                    c[i - 1, j - 1] = 1.0 / (jf - jm) * (jf - i)
    elif nj == nz:
        c[:, :] = np.eye(nz)
    else:
        raise ValueError("NJ cannot be larger than NZ")
    return c


def weights(numw, wstk=(1.0, 1.0, 1.0, 1.0), isigma=4.0e-3):
    """ISIGMAP(NFREQ) for all four Stokes parameters inverted."""
    w = np.array(wstk, dtype=np.float32)
    minw = np.float32(np.sqrt(np.sum(w.astype(np.float32) ** 2)) / np.sqrt(np.float32(4.0)))
    w = (w / minw).astype(np.float32)
    return np.repeat(w.astype(np.float64) ** 2 / isigma ** 2, numw)


def update_lambda(chicur, chipre, lam, steps, precyc, factor=0.01):
    """UPDATE_LAMBDA; returns (chipre, lam, steps, precyc)."""
    lmin = 1.0e-2
    if chipre - chicur > 0:
        if chipre - chicur > factor * chipre:
            steps = max(0.0, steps - 1.0)
        else:
            steps = steps + 1.0
        chipre = chicur
        lam = lam / np.sqrt(10.0)
    else:
        if abs(precyc - 1.0) < 1.0e-2:
            precyc = 0.0
            lam = lam * 3.0
        else:
            lam = lam * 10.0
        steps = steps + 1.0
    return chipre, max(lmin, lam), steps, precyc


def pinv_dgesvd(m, svdtol=RSVDTOL):
    """GET_INVERSE (src/lm.f90:61-133): DGESVD pseudo-inverse, singular
    values below svdtol * max dropped."""
    u, s, vt, info = lapack.dgesvd(np.asfortranarray(m), full_matrices=True)
    if info != 0:
        raise RuntimeError("dgesvd info %d" % info)
    thr = np.max(np.abs(s)) * svdtol
    si = np.where(np.abs(s) < thr, 0.0, 1.0 / np.where(s == 0, 1.0, s))
    return vt.T @ (np.diag(si) @ u.T)


def cg_delta(a, b):
    """NEW_CALCULATE_DELTA_UBICGSTAB (src/lm.f90:375-453): conjugate
    gradients from x = 0 until mean(((A x - b)/(|b| + 1e-5))^2) < 1e-3 (or
    the measure grows by more than 1e30), at most 100000 iterations; x / 10
    when it does not converge (a non-finite measure gives up at once: its
    result is non-finite either way)."""
    npar = b.size
    x = np.zeros(npar)
    p = b.copy()
    r = b - a @ x
    rho = float(r @ r)
    q = a @ p
    alpha = rho / float(p @ q)
    x = x + alpha * p
    r = r - alpha * q
    pc, dc = 1.0e29, -1.0e29
    with np.errstate(all="ignore"):
        for _ in range(100000):
            rho0 = rho
            rho = float(r @ r)
            beta = rho / rho0
            p = r + beta * p
            q = a @ p
            alpha = rho / float(p @ q)
            x = x + alpha * p
            r = r - alpha * q
            cond = float(np.sum(((a @ x - b) / (np.abs(b) + 1.0e-5)) ** 2)) / npar
            if cond < 1.0e-3 or dc > 1.0e30:
                return x
            if cond != cond:
                break
            dc = cond - pc
            pc = cond
    return x / 10.0


def get_perturbation(jac_n, diff, lam, svdtol=RSVDTOL, reg_pen=None, reg_hss=None, dtype=1):
    """GET_PERTURBATION (src/lm.f90:137-204), DTYPE 1 (SVD) or 2 (conjugate
    gradients): jac_n is the normalised JACOB (NFREQ, NP), diff the weighted
    residual; REG_PEN is subtracted from J^T diff and REG_HSS added to J^T J
    (:170-174)."""
    hss = jac_n.T @ jac_n
    term2 = jac_n.T @ diff
    if reg_pen is not None:
        term2 = term2 - reg_pen
    if reg_hss is not None:
        hss = hss + reg_hss
    term1 = hss.copy()
    term1[np.diag_indices_from(term1)] += np.diag(hss) * lam
    delta = cg_delta(term1, term2) if dtype == 2 else pinv_dgesvd(term1, svdtol) @ term2
    return np.where(np.isnan(delta), 0.0, delta)


def contract(ivec_sp, coefs):
    """CONTRACT_VECTOR: node averages of a REAL*4 height profile."""
    o = (ivec_sp.astype(np.float32).astype(np.float64)[:, None] * coefs).sum(axis=0)
    return o / coefs.sum(axis=0)


def expand(ivec, coefs):
    """EXPAND_VECTOR."""
    return coefs @ ivec


def sort_delta(delta, factor, ipar, inf, sup, coefs, absolute, node_expansion=1):
    """SORT_DELTA_TO_ATMOSPHERE with NODE_EXPANSION = 1 (SIR-like) or 2
    (STiC-like, :1792-1804): returns the REAL*4 height perturbation of one
    parameter (and the clipped node deltas)."""
    itd = delta * factor
    avg = contract(ipar, coefs)
    pert = np.maximum(absolute, np.abs(MPERT * avg)) if absolute > 0 else np.abs(MPERT * avg)
    pert = np.where(avg == 0, absolute, pert)
    itd = np.where(np.abs(itd) > pert, itd / np.abs(np.where(itd == 0, 1.0, itd)) * pert, itd)
    nzpert = expand(avg + itd, coefs)
    if node_expansion == 2:
        opar = nzpert.astype(np.float32)
        opar = np.where(opar.astype(np.float64) < inf, np.float32(inf), opar)
        opar = np.where(opar.astype(np.float64) > sup, np.float32(sup), opar)
        return (opar - ipar.astype(np.float32)).astype(np.float32), itd
    nzpert = nzpert - ipar.astype(np.float64)
    itd = contract(nzpert.astype(np.float32), coefs)
    nzpert = expand(itd, coefs)
    opar = (ipar + nzpert.astype(np.float32)).astype(np.float32)
    nzpert = np.where(opar < inf, inf - ipar.astype(np.float64), nzpert)
    nzpert = np.where(opar > sup, sup - ipar.astype(np.float64), nzpert)
    return nzpert.astype(np.float32), itd


def rearange(model, delta, nodes, node_expansion=1):
    """REARANGE_DA_MODEL (non-errors limits): applies the node perturbation
    delta to model (13, NZ) REAL*4 in place.  nodes: {param: NJ}."""
    nz = model.shape[1]
    j0 = 0
    for p in range(1, 9):
        nj = nodes.get(p, 0)
        if nj <= 0:
            continue
        row = ATMPOS[p]
        coefs = int_coefs(nz, nj)
        bumod = model[row].copy()
        pert, _ = sort_delta(delta[j0:j0 + nj], PARAM_NORMS[p - 1], model[row], LOWLIM[p - 1], UPPLIM[p - 1],
                             coefs, PARAM_NORMS[p - 1] * MPERT, node_expansion)
        if p == 1:
            tll, tul = np.float32(-11.5), np.float32(0.5)
            tau = model[TAU_ROW]
            for k in range(nz - 1, -1, -1):
                if tau[k] < tll:
                    pert[k] = np.float32(np.exp(np.float32(-(np.float32(abs(tau[k] - tll)) / np.float32(0.5)) ** 2))) * pert[k]
                elif tau[k] > tul and k + 1 < nz:
                    pert[k] = pert[k + 1]
        model[row] = (pert + bumod).astype(np.float32)
        j0 += nj


def it_penalties(model, nodes, pen_typ, pen_alp):
    """GET_IT_PENALTIES (src/get_dmodel.f90:1041-1197) on model (13, NZ): per
    free parameter p the node values x = CONTRACT_VECTOR(row) / PARAM_NORM, the
    operator L = ALP D with ALP = sqrt(PEN_ALP / IFREEP) and D = diag(1/NJ)
    (type 0) or first differences to the previous node (type 1, first row
    zero); returns (PEN_RES = L^T L x, PEN_HSS = L^T L), block diagonal over
    the parameters in node order.  pen_typ, pen_alp: per reference parameter
    1..8."""
    nz = model.shape[1]
    npar = sum(n for n in nodes.values() if n > 0)
    res = np.zeros(npar)
    hss = np.zeros((npar, npar))
    j0 = 0
    for p in range(1, 9):
        nj = nodes.get(p, 0)
        if nj <= 0:
            continue
        x = contract(model[ATMPOS[p]], int_coefs(nz, nj)) / PARAM_NORMS[p - 1]
        lop = np.zeros((nj, nj))
        if pen_typ[p - 1] == 0:
            lop[np.diag_indices(nj)] = 1.0 / nj
        elif pen_typ[p - 1] == 1:
            for k in range(1, nj):
                lop[k, k] = 1.0
                lop[k, k - 1] = -1.0
        lop *= np.sqrt(float(pen_alp[p - 1]) / float(npar))
        res[j0:j0 + nj] = lop.T @ (lop @ x)
        hss[j0:j0 + nj, j0:j0 + nj] = lop.T @ lop
        j0 += nj
    return res, hss


def normalize_jacob(jac, w, inu, nodes):
    """NORMALIZE_JACOB: JACOB (NFREQ, NP) REAL*8 of the REAL*4 EQVDSYN."""
    j = jac.astype(np.float64) * (np.sqrt(w) / np.sqrt(inu))[:, None]
    c = 0
    for p in range(1, 9):
        nj = nodes.get(p, 0)
        if nj > 0:
            j[:, c:c + nj] *= PARAM_NORMS[p - 1]
            c += nj
    return j


class PixelState:
    """INV_SLA(1:9) of one pixel plus its best/current model, synthesis and
    Jacobian (INITIALIZE_CYCLE, src/invert3d.f90:275-286)."""

    def __init__(self, model):
        self.steps, self.chicur, self.chibest, self.precyc, self.lam = 0.0, 1.0e29, 1.0e29, 0.0, 10.0
        self.cur = np.array(model, dtype=np.float32)
        self.best = self.cur.copy()
        self.best_syn = None
        self.best_jac = None


def lm_accept(st, obs, syn, jac, w, ok=True, reg=None):
    """NEW_CALCULATE_CHI2 + UPDATE_LAMBDA for one pixel; returns (chi, accepted,
    previous best chi).  reg = (nodes, pen_typ, pen_alp): the penalty of the
    current model, sum(PEN_RES^2), is added to chi2 (:966-983)."""
    inu = float(obs.size)
    chi = float(np.sum((obs - syn) ** 2 * w) / inu) if ok else 1.0e300
    if reg is not None and ok:
        pen, _ = it_penalties(st.cur, *reg)
        chi += float(np.sum(pen * pen))
    prev = st.chibest
    st.chicur = chi
    acc = chi < st.chibest
    if acc:
        st.best = st.cur.copy()
        st.best_jac = jac.copy()
        st.best_syn = syn.copy()
    else:
        st.cur = st.best.copy()
    st.chibest, st.lam, st.steps, st.precyc = update_lambda(chi, st.chibest, st.lam, st.steps, st.precyc, 0.01)
    return chi, acc, prev


def lm_perturb(st, obs, w, nodes, reg=None, solver=1, node_expansion=1):
    """The rest of GET_PERT_1D: normalised Jacobian, GET_PERTURBATION (with the
    penalties of the best model, reg as in lm_accept) and REARANGE_DA_MODEL;
    st.cur becomes the next trial model."""
    inu = float(obs.size)
    diff = (obs - st.best_syn) * np.sqrt(w) / np.sqrt(inu)
    jn = normalize_jacob(st.best_jac, w, inu, nodes)
    pen = hss = None
    if reg is not None:
        pen, hss = it_penalties(st.best, *reg)
    delta = get_perturbation(jn, diff, st.lam, reg_pen=pen, reg_hss=hss, dtype=solver)
    rearange(st.cur, delta, nodes, node_expansion)
    return delta


def lm_step(st, obs, syn, jac, w, nodes):
    """GET_PERT_1D for one pixel (syn/jac: forward synthesis and EQVDSYN of
    st.cur, obs/syn RSYN1D(NFREQ), jac (NFREQ, NP) REAL*4)."""
    lm_accept(st, obs, syn, jac, w)
    return lm_perturb(st, obs, w, nodes)


def invert(forward_rf, obs, init, nodes, w, maxsteps=5, maxit=40, dchi2=0.0, reg=None, solver=1,
           node_expansion=1, record=None):
    """Pixel-wise inversion with the stop rules of the batched GPU inversion
    (steps > maxsteps, maxit iterations, or an accepted step gaining less than
    dchi2 relative).  forward_rf(models (n,13,nz)) -> (syn (n,nfreq),
    jac (n,nfreq,np), models_out, status); obs (npix, nfreq); reg =
    (pen_typ, pen_alp) per reference parameter adds the vertical
    regularisation of GET_IT_PENALTIES.  record: a list that receives, per
    iteration k (record[k-1], a dict by pixel), each pixel's state right after
    that iteration's accept step -- (STEPS, chi2 of the model just
    synthesised, best chi2, PRECYC, lambda, best model, accepted) -- which is
    the final state of the same inversion stopped at maxit = k.  Returns (best
    models, chi2, iterations)."""
    if reg is not None:
        reg = (nodes,) + tuple(reg)
    npix = obs.shape[0]
    states = [PixelState(init[i]) for i in range(npix)]
    iters = np.zeros(npix, dtype=np.int32)
    active = list(range(npix))
    while active:
        models = np.stack([states[i].cur for i in active])
        syn, jac, mo, status = forward_rf(models)
        still = []
        for a, i in enumerate(active):
            st = states[i]
            st.cur = mo[a].copy()
            _, acc, prev = lm_accept(st, obs[i], syn[a], jac[a], w, ok=status[a] == 0, reg=reg)
            iters[i] += 1
            if record is not None:
                while len(record) < iters[i]:
                    record.append({})
                record[iters[i] - 1][i] = (st.steps, st.chicur, st.chibest, st.precyc, st.lam, st.best.copy(), acc)
            small = acc and prev < 1.0e29 and (prev - st.chibest) < dchi2 * prev
            if st.steps > maxsteps or iters[i] >= maxit or small:
                continue
            lm_perturb(st, obs[i], w, nodes, reg=reg, solver=solver, node_expansion=node_expansion)
            still.append(i)
        active = still
    best = np.stack([st.best for st in states])
    chi = np.array([st.chibest for st in states])
    return best, chi, iters


def smoothing_b(models, nx, ny, params):
    """SMOOTHING_B (src/model_spatial_extension.f90:351-491): models
    (NY*NX, 13, NZ) REAL*4 with pixel iy + NY*ix; for every reference
    parameter in params (1..8; 8 = P0 smooths Pg) the cube is taken to REAL*8,
    averaged 1-2-1 along x, then y, then z (array assignments: each pass
    reads the previous pass's whole array; first and last points of a
    direction kept; a direction of 4 or fewer points skipped) and rounded
    back to REAL*4.  The kernel built with FFTW in the routine never touches
    the model."""
    m = np.array(models, dtype=np.float32, copy=True)
    nz = m.shape[2]
    for p in params:
        row = ATMPOS[p] if p != 8 else 1
        a = m[:, row, :].astype(np.float64).reshape(nx, ny, nz)
        if nx > 4:
            a[1:-1] = (a[2:] + a[:-2] + a[1:-1] * 2.0) / 4.0
        if ny > 4:
            a[:, 1:-1] = (a[:, 2:] + a[:, :-2] + a[:, 1:-1] * 2.0) / 4.0
        if nz > 4:
            a[:, :, 1:-1] = (a[:, :, 2:] + a[:, :, :-2] + a[:, :, 1:-1] * 2.0) / 4.0
        m[:, row, :] = a.reshape(nx * ny, nz).astype(np.float32)
    return m


def errors_1d(obs, syn, jac, model, w, nodes, reg=None):
    """GET_ERROR_1D (src/get_dmodel.f90:1248-1287) for one pixel: obs, syn
    RSYN1D (NFREQ,); jac EQVDSYN (NFREQ, NP) REAL*4 of model (13, NZ); reg =
    (pen_typ, pen_alp) adds the current model's penalties to chi2 as
    NEW_CALCULATE_CHI2 does (:966-983).  NEW_SOLVE_ERRORS (:1291-1323):
    NUME = chi2 / INU, H = HESSIAN of the normalised Jacobian, sigma_i =
    sqrt(NUME / H_ii) where H_ii > 1e-32, else 1e32 (its GET_INVERSE_COV
    result is unused).  LIMIT_PERTURBATION with ERRORS on MODEL = 0:
    REARANGE_DA_MODEL's errors limits LOWLIM = 0, UPPLIM = 1e20 (:1877-1883).
    Returns (err (13, NZ) REAL*4, chi2)."""
    inu = float(obs.size)
    chi = float(np.sum((obs - syn) ** 2 * w) / inu)
    if reg is not None:
        pen, _ = it_penalties(model, nodes, *reg)
        chi += float(np.sum(pen * pen))
    jn = normalize_jacob(jac, w, inu, nodes)
    hd = np.einsum("fi,fi->i", jn, jn)
    nume = chi / inu
    sig = np.where(hd > 1.0e-32, np.sqrt(nume / np.where(hd > 0, hd, 1.0)), 1.0e32)
    nz = model.shape[1]
    err = np.zeros((13, nz), dtype=np.float32)
    j0 = 0
    for p in range(1, 9):
        nj = nodes.get(p, 0)
        if nj <= 0:
            continue
        row = ATMPOS[p]
        coefs = int_coefs(nz, nj)
        pert, _ = sort_delta(sig[j0:j0 + nj], PARAM_NORMS[p - 1], err[row], 0.0, 1.0e20, coefs,
                             PARAM_NORMS[p - 1] * MPERT)
        # the T taper reads log tau5 of the zeroed model: 0 lies inside
        # (-11.5, 0.5], so the profile is kept
        err[row] = (pert + err[row]).astype(np.float32)
        j0 += nj
    return err, chi


def smoothing_b_shard(models, nx, ny, x0, nx_field, params):
    """SMOOTHING_B of a shard: models (nx*ny, 13, NZ) hold field columns
    x0 .. x0+nx-1 (halo columns included) of an nx_field-column field; the x
    pass applies to the field's interior columns that have both neighbours
    in the array, the field's own 4-point rule decides; y and z as
    smoothing_b.  The interior columns match smoothing_b of the whole field."""
    m = np.array(models, dtype=np.float32, copy=True)
    nz = m.shape[2]
    for p in params:
        row = ATMPOS[p] if p != 8 else 1
        a = m[:, row, :].astype(np.float64).reshape(nx, ny, nz)
        if nx_field > 4:
            b = a.copy()
            for ix in range(1, nx - 1):
                gx = ix + x0
                if 0 < gx < nx_field - 1:
                    b[ix] = (a[ix + 1] + a[ix - 1] + a[ix] * 2.0) / 4.0
            a = b
        if ny > 4:
            a[:, 1:-1] = (a[:, 2:] + a[:, :-2] + a[:, 1:-1] * 2.0) / 4.0
        if nz > 4:
            a[:, :, 1:-1] = (a[:, :, 2:] + a[:, :, :-2] + a[:, :, 1:-1] * 2.0) / 4.0
        m[:, row, :] = a.reshape(nx * ny, nz).astype(np.float32)
    return m
