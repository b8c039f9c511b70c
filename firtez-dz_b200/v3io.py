"""FIRTEZ-dz v3 files: the model atmosphere, Stokes profile and response
function files the reference's Fortran host and Python module read and
write (src/misc.f90 READ_MODEL_3D, WRITE_MODEL3D_V3, READ_PROFILE_3D,
WRITE_PROFILES3D_V3, WRITE_RFS3D_V3; python/firtez_dz.py read_model,
read_profile, read_rf), and the GPU layout changes between them and the
library's device arrays.

File arrays are the file's own order, in C terms:
  model cubes  (13, NX, NY, NZ): T, Pg, rho, Bx, By, Bz, vz, Pe, mu,
               log tau5, x, y, z
  profiles     (NX, NY, NW, 4)
  RFs          (NX, NY, NZ, NW, 4, NPAR), NPAR = the LOGV-flagged of T, Pg,
               rho, Bx, By, Bz, vz, P0
Device arrays: MODEL (npix, 13, NZ), OBS3D / RSYN1D (npix, 4, NW) float64,
fz_forward_rf_full output (npix, 6, NZ, 4 NW); pixel index iy + NY ix.
"""
import ctypes

import numpy as np

from . import FzError, _check, _p, lib

MODEL_ID, PROFILE_ID, RF_ID = 130904, 160904, 18060904


def _path(path):
    return str(path).encode()


def read_header(path):
    """(ID, version, dims) of a v3 file."""
    fid, ver, nd = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    dims = np.zeros(8, dtype=np.int32)
    _check(lib().fz_v3_header(_path(path), ctypes.byref(fid), ctypes.byref(ver), ctypes.byref(nd), _p(dims)))
    return fid.value, ver.value, tuple(int(d) for d in dims[:nd.value])


def read_model(path):
    """Model cubes (13, NX, NY, NZ) float32 of a v3 model file."""
    fid, ver, dims = read_header(path)
    if fid != MODEL_ID or ver != 3 or len(dims) != 4:
        raise FzError("%s: not a v3 model file" % path)
    _, nx, ny, nz = dims
    cubes = np.empty((13, nx, ny, nz), dtype=np.float32)
    _check(lib().fz_v3_read_model(_path(path), nx, ny, nz, _p(cubes)))
    return cubes


def write_model(path, cubes):
    c = np.ascontiguousarray(cubes, dtype=np.float32)
    if c.ndim != 4 or c.shape[0] != 13:
        raise ValueError("cubes must be (13, nx, ny, nz)")
    _check(lib().fz_v3_write_model(_path(path), c.shape[1], c.shape[2], c.shape[3], _p(c)))


def read_profile(path):
    """(ind, wave, stokes (NX, NY, NW, 4) float32) of a v3 profile file."""
    fid, ver, dims = read_header(path)
    if fid != PROFILE_ID or ver != 3 or len(dims) != 4:
        raise FzError("%s: not a v3 profile file" % path)
    nx, ny, nw, _ = dims
    ind = np.empty(nw, dtype=np.float32)
    wave = np.empty(nw, dtype=np.float32)
    st = np.empty((nx, ny, nw, 4), dtype=np.float32)
    _check(lib().fz_v3_read_profiles(_path(path), nx, ny, nw, _p(ind), _p(wave), _p(st)))
    return ind, wave, st


def write_profile(path, ind, wave, stokes):
    st = np.ascontiguousarray(stokes, dtype=np.float32)
    if st.ndim != 4 or st.shape[3] != 4:
        raise ValueError("stokes must be (nx, ny, nw, 4)")
    nx, ny, nw, _ = st.shape
    i = np.ascontiguousarray(ind, dtype=np.float64)
    w = np.ascontiguousarray(wave, dtype=np.float64)
    if i.size != nw or w.size != nw:
        raise ValueError("ind and wave must have nw entries")
    _check(lib().fz_v3_write_profiles(_path(path), nx, ny, nw, _p(i), _p(w), _p(st)))


def read_rf(path):
    """(z, logv (8,), ind, wave, data (NX, NY, NZ, NW, 4, NPAR)) of a v3 RF file."""
    fid, ver, dims = read_header(path)
    if fid != RF_ID or ver != 3 or len(dims) != 6:
        raise FzError("%s: not a v3 response-function file" % path)
    nx, ny, nz, nw, _, _ = dims
    z = np.empty(nz, dtype=np.float32)
    ind = np.empty(nw, dtype=np.float32)
    wave = np.empty(nw, dtype=np.float32)
    logv = np.zeros(8, dtype=np.int32)
    npar = _check(lib().fz_v3_read_rfs(_path(path), nx, ny, nz, nw, _p(z), _p(logv), _p(ind), _p(wave), None))
    data = np.empty((nx, ny, nz, nw, 4, npar), dtype=np.float32)
    _check(lib().fz_v3_read_rfs(_path(path), nx, ny, nz, nw, _p(z), _p(logv), _p(ind), _p(wave), _p(data)))
    return z, logv, ind, wave, data


def write_rf(path, z, logv, ind, wave, data):
    d = np.ascontiguousarray(data, dtype=np.float32)
    lv = np.ascontiguousarray([1 if v else 0 for v in logv], dtype=np.int32)
    if d.ndim != 6 or d.shape[4] != 4 or lv.size != 8 or d.shape[5] != int(lv.sum()):
        raise ValueError("data must be (nx, ny, nz, nw, 4, sum(logv))")
    nx, ny, nz, nw = d.shape[:4]
    zz = np.ascontiguousarray(z, dtype=np.float64)
    i = np.ascontiguousarray(ind, dtype=np.float64)
    w = np.ascontiguousarray(wave, dtype=np.float64)
    _check(lib().fz_v3_write_rfs(_path(path), nx, ny, nz, nw, _p(zz), _p(lv), _p(i), _p(w), _p(d)))


def read_lsf(path, n):
    """The n-point line spread function of an LSF file (READ_LSF_FILE)."""
    yk = np.empty(n, dtype=np.float64)
    _check(lib().fz_v3_read_lsf(_path(path), int(n), _p(yk)))
    return yk


def write_lsf(path, yk):
    k = np.ascontiguousarray(yk, dtype=np.float64)
    _check(lib().fz_v3_write_lsf(_path(path), k.size, _p(k)))


# ---------------------------------------------------------------- device
def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    return ctypes.c_void_p(stream) if stream else None


def model_from_cubes_device(d_cubes, out=None, stream=0):
    """MODEL (npix, 13, NZ) on the device from model cubes (13, NX, NY, NZ)
    already on the device (torch tensors)."""
    import torch
    _, nx, ny, nz = d_cubes.shape
    out = out if out is not None else torch.empty((nx * ny, 13, nz), dtype=torch.float32, device=d_cubes.device)
    _check(lib().fz_model_from_v3_device(nx, ny, nz, _ptr(d_cubes.contiguous()), _ptr(out), _stream(stream)))
    return out


def cubes_from_model_device(d_model, nx, ny, x, y, out=None, stream=0):
    """Model cubes (13, NX, NY, NZ) on the device from MODEL (npix, 13, NZ);
    x (NX,), y (NY,) host coordinate vectors."""
    import torch
    nz = d_model.shape[2]
    out = out if out is not None else torch.empty((13, nx, ny, nz), dtype=torch.float32, device=d_model.device)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    yy = np.ascontiguousarray(y, dtype=np.float64)
    _check(lib().fz_model_to_v3_device(nx, ny, nz, _ptr(d_model), _p(xx), _p(yy), _ptr(out), _stream(stream)))
    return out


def obs_from_stokes_device(d_stokes, out=None, stream=0):
    """OBS3D (npix, 4, NW) float64 from profiles (NX, NY, NW, 4) float32."""
    import torch
    nx, ny, nw, _ = d_stokes.shape
    out = out if out is not None else torch.empty((nx * ny, 4, nw), dtype=torch.float64, device=d_stokes.device)
    _check(lib().fz_obs_from_v3_device(nx * ny, nw, _ptr(d_stokes.contiguous()), _ptr(out), _stream(stream)))
    return out


def stokes_from_syn_device(d_syn, nx, ny, out=None, stream=0):
    """Profiles (NX, NY, NW, 4) float32 from RSYN1D (npix, 4, NW) float64."""
    import torch
    nw = d_syn.shape[2]
    out = out if out is not None else torch.empty((nx, ny, nw, 4), dtype=torch.float32, device=d_syn.device)
    _check(lib().fz_syn_to_v3_device(nx * ny, nw, _ptr(d_syn.contiguous()), _ptr(out), _stream(stream)))
    return out


def rf_file_layout_device(d_rf, nx, ny, out=None, stream=0):
    """The RF file payload (NX, NY, NZ, NW, 4, 6) from fz_forward_rf_full's
    (npix, 6, NZ, 4 NW) output (LOGV: T, Pg, Bx, By, Bz, vz)."""
    import torch
    npix, _, nz, nf = d_rf.shape
    nw = nf // 4
    out = out if out is not None else torch.empty((nx, ny, nz, nw, 4, 6), dtype=torch.float32, device=d_rf.device)
    _check(lib().fz_rf_to_v3_device(npix, nz, nw, _ptr(d_rf.contiguous()), _ptr(out), _stream(stream)))
    return out


RF_FULL_LOGV = (1, 1, 0, 1, 1, 1, 1, 0)
