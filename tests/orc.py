"""ctypes wrapper of the FP64 CPU oracle (oracle/liborc.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, as the checker.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "liborc.so")

MAXBLEND = 8

LINE_DTYPE = np.dtype([
    ("num", "<i4"), ("zn", "<i4"), ("ion", "<i4"), ("flag", "<i4"), ("otr", "<i4", 2),
    ("abo_ierr", "<i4"), ("pad", "<i4"),
    ("l0", "<f8"), ("loggf", "<f8"), ("eplow", "<f8"), ("alpha", "<f8"), ("sigma", "<f8"),
    ("sl", "<f8"), ("ll", "<f8"), ("jl", "<f8"), ("su", "<f8"), ("lu", "<f8"), ("ju", "<f8"),
    ("elowlim", "<f8"), ("eupplim", "<f8"),
], align=True)

REGION_DTYPE = np.dtype([
    ("nblend", "<i4"), ("line", "<i4", MAXBLEND), ("wdif", "<f8", MAXBLEND),
    ("numwave", "<i4"), ("pad", "<i4"), ("wave_ini", "<f8"), ("dlambda", "<f8"),
], align=True)

_lib = None


def build():
    import subprocess
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.orc_partition.argtypes = [ctypes.c_int, ctypes.c_double, P]
        L.orc_get_rho.argtypes = [ctypes.c_double, ctypes.c_double, P, P]
        L.orc_opac_continuum.argtypes = [ctypes.c_float, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_opac_continuum.restype = ctypes.c_double
        L.orc_parse_lines.argtypes = [ctypes.c_char_p, P, ctypes.c_int]
        L.orc_zeeman.argtypes = [P, P, P, P, ctypes.c_int]
        L.orc_voigt.argtypes = [ctypes.c_int, ctypes.c_double, P, P, P]
        L.orc_rte_solve.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P, P]
        L.orc_gain.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P]
        L.orc_forward.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int, P,
                                  ctypes.c_int, P, P, ctypes.c_int]
        L.orc_set_abundances.argtypes = [P]
        L.orc_forward_rf.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int, P,
                                     ctypes.c_int, P, P, P, P, ctypes.c_int]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def set_abundances(ab=None):
    if ab is None:
        lib().orc_set_abundances(None)
    else:
        ab = np.ascontiguousarray(ab, dtype=np.float64)
        lib().orc_set_abundances(_p(ab))


def partition(zn, T):
    out = np.zeros(6)
    lib().orc_partition(int(zn), float(T), _p(out))
    return out


def get_rho(T, pg, nelec=0.0):
    ne = np.array([nelec], dtype=np.float64)
    out = np.zeros(5)
    st = lib().orc_get_rho(float(T), float(pg), _p(ne), _p(out))
    return dict(nhyd=out[0], pelec=out[1], dens=out[2], molecw=out[3], iters=int(out[4]), nelec=ne[0], status=st)


def parse_lines(text):
    out = np.zeros(512, dtype=LINE_DTYPE)
    n = lib().orc_parse_lines(text.encode(), _p(out), len(out))
    if n < 0:
        raise ValueError("line database parse failed (%d)" % n)
    return out[:n].copy()


def regions(section, lines):
    """REGION_DTYPE rows of a LINES: section (src/input_file.f90:290-366):
    ``ids numwave wave_ini dlambda`` per row, ids comma-separated database
    numbers of the main line and its blends; BLENDSDIFF = 1e3 (lambda_blend -
    lambda_main) mA (:346-354)."""
    pos = {int(n): i for i, n in enumerate(lines["num"])}
    rows = [r.split() for r in section.strip().splitlines() if r.strip() and not r.strip().startswith("#")]
    out = np.zeros(len(rows), dtype=REGION_DTYPE)
    for k, f in enumerate(rows):
        ids = [int(x) for x in f[0].split(",") if x]
        if not ids or len(ids) > MAXBLEND or any(i not in pos for i in ids):
            raise ValueError("LINES row %r" % " ".join(f))
        out["nblend"][k] = len(ids)
        for b, i in enumerate(ids):
            out["line"][k, b] = pos[i]
            out["wdif"][k, b] = 1.0e3 * (lines["l0"][pos[i]] - lines["l0"][pos[ids[0]]]) if b else 0.0
        out["numwave"][k], out["wave_ini"][k], out["dlambda"][k] = int(f[1]), float(f[2]), float(f[3])
    return out


def zeeman(line):
    ln = np.ascontiguousarray(np.array(line, dtype=LINE_DTYPE).reshape(1))
    sh, st, ty = np.zeros(64), np.zeros(64), np.zeros(64, dtype=np.int32)
    n = lib().orc_zeeman(_p(ln), _p(sh), _p(st), _p(ty), 64)
    return sh[:n], st[:n], ty[:n]


def voigt(a, v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    h, f = np.zeros_like(v), np.zeros_like(v)
    lib().orc_voigt(len(v), float(a), _p(v), _p(h), _p(f))
    return h, f


def rte_solve(eta, src, zz, bnd=None):
    """SET_BOUNDARY + OLD_ANALYTICAL_SOLVER on given matrices: eta (nz, 7,
    nw) ETAI..RHOV [cm^-1], src (nz, nw), zz (nz) km, bnd (nz) or None.
    Returns SYN1D as (nw, 4)."""
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    nz, _, nw = eta.shape
    src = np.ascontiguousarray(src, dtype=np.float64)
    zz = np.ascontiguousarray(zz, dtype=np.float64)
    b = None if bnd is None else np.ascontiguousarray(bnd, dtype=np.int32)
    out = np.zeros((nw, 4))
    lib().orc_rte_solve(nz, nw, _p(eta), _p(src), _p(zz), None if b is None else _p(b), _p(out))
    return out


def gain(lines, regions):
    lines = np.ascontiguousarray(lines, dtype=LINE_DTYPE)
    regions = np.ascontiguousarray(regions, dtype=REGION_DTYPE)
    numw = int(regions["numwave"].sum())
    g = np.zeros((numw, 4), dtype=np.float32)
    st = lib().orc_gain(_p(lines), len(lines), _p(regions), len(regions), _p(g))
    return g, st


def forward(lines, regions, gain_, model, hydrostatic=False, nthreads=0):
    """model: (ncol, 13, nz) float32 (C order == Fortran MODEL(NZ,13,ncol)).

    Returns (stokes (ncol, 4, numw) float64, model_out, status)."""
    lines = np.ascontiguousarray(lines, dtype=LINE_DTYPE)
    regions = np.ascontiguousarray(regions, dtype=REGION_DTYPE)
    g = np.ascontiguousarray(gain_, dtype=np.float32)
    m = np.array(model, dtype=np.float32, order="C", copy=True)
    ncol, npar, nz = m.shape
    assert npar == 13
    numw = int(regions["numwave"].sum())
    stokes = np.zeros((ncol, 4, numw))
    status = np.zeros(ncol, dtype=np.int32)
    lib().orc_forward(_p(lines), len(lines), _p(regions), len(regions), _p(g), nz, ncol, _p(m),
                      int(hydrostatic), _p(stokes), _p(status), int(nthreads))
    return stokes, m, status


# reference parameter index (1-based) -> name, as in src/atm_param.f90 order
RF_PARAMS = {1: "T", 2: "Pg", 4: "Bx", 5: "By", 6: "Bz", 7: "vz"}


def forward_rf(lines, regions, gain_, model, nodes, hydrostatic=False, nthreads=0):
    """FORWARD1D with response functions.

    nodes: dict {reference parameter index: node count} (1 T, 2 Pg, 4 Bx,
    5 By, 6 Bz, 7 vz).  Returns (stokes (ncol,4,numw), jac (ncol, NP, 4*numw)
    float32 = EQVDSYN transposed per column, model_out, status)."""
    lines = np.ascontiguousarray(lines, dtype=LINE_DTYPE)
    regions = np.ascontiguousarray(regions, dtype=REGION_DTYPE)
    g = np.ascontiguousarray(gain_, dtype=np.float32)
    m = np.array(model, dtype=np.float32, order="C", copy=True)
    ncol, npar, nz = m.shape
    numw = int(regions["numwave"].sum())
    nv = np.zeros(8, dtype=np.int32)
    for p, n in nodes.items():
        nv[p - 1] = n
    np_ = int(nv.sum())
    stokes = np.zeros((ncol, 4, numw))
    jac = np.zeros((ncol, np_, 4 * numw), dtype=np.float32)
    status = np.zeros(ncol, dtype=np.int32)
    r = lib().orc_forward_rf(_p(lines), len(lines), _p(regions), len(regions), _p(g), nz, ncol, _p(m),
                             int(bool(hydrostatic)), _p(nv), _p(stokes), _p(jac), _p(status), int(nthreads))
    if r < 0:
        raise ValueError("orc_forward_rf rejected the node set (%d)" % r)
    return stokes, jac, m, status
