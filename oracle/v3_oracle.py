"""TEST INFRASTRUCTURE -- not part of the product.

numpy restatement of FIRTEZ-dz's v3 files and of the array layouts the
Fortran host builds from them, used by tests/ as the checker of the C++
record I/O (firtez-dz_b200/csrc/fz_io.cpp) and of the GPU layout kernels.

Followed (src/ unless noted):
  records     Fortran unformatted sequential (4-byte little-endian byte
              counts around each REAL*4 payload); data records of at most
              NMAXREC = 268,435,446 values (misc.f90:16-17)
  model       WRITE_MODEL3D_V3 misc.f90:801-929, READ_MODEL_3D :374-499
              (header 3003, 2997, 130904, NRECS+1, 4, 13, NX, NY, NZ; cubes
              (NZ,NY,NX) of T, Pg, rho, Bx, By, Bz, vz, Pe, mu, log tau5, x, y, z)
  profiles    WRITE_PROFILES3D_V3 :1147-1249 (header 3003, 2997, 160904,
              NRECS+3, 4, NX, NY, NW, 4; IND, WAVE; STOKES(4,NW,NY,NX))
  RFs         WRITE_RFS3D_V3 :1862-1999 (header 3003, 2997, 18060904,
              NRECS+5, 6, NX, NY, NZ, NW, 4, 8; Z, IND, WAVE, LOGV;
              DSTOKES(P,4,NW,NZ,NY,NX) over the LOGV-flagged parameters)
  MODEL rows  JOIN_MODEL2 forward.f90:363-405 (T, Pg, rho, Pe, mu, Bx, By, Bz,
              vx, vy, vz, log tau5, z; ZZ = the first pixel's z column)
  OBS3D       ALLOCATE_AND_READ pre_post_duties.f90:421-431 (Stokes-major
              blocks of NW per pixel, REAL*8 of the file's REAL*4)
  WDSYN       WRITE_RESPONSE_FUNCTIONS pre_post_duties.f90:316-356
"""
import struct

import numpy as np

NMAXREC = 1073741784 // 4
# file cube of each MODEL row (None: vx, vy -- not in the file)
CUBE_OF_ROW = [0, 1, 2, 7, 8, 3, 4, 5, None, None, 6, 9, 12]
ROW_OF_CUBE = [0, 1, 2, 5, 6, 7, 10, 3, 4, 11]


def read_records(path):
    """All records of a Fortran unformatted sequential file as float32 arrays."""
    b = open(path, "rb").read()
    off, out = 0, []
    while off < len(b):
        n = struct.unpack("<i", b[off:off + 4])[0]
        out.append(np.frombuffer(b[off + 4:off + 4 + n], dtype="<f4").copy())
        if struct.unpack("<i", b[off + 4 + n:off + 8 + n])[0] != n:
            raise ValueError("record markers differ")
        off += 8 + n
    return out


def record_bytes(arrays):
    out = b""
    for a in arrays:
        a = np.ascontiguousarray(a, dtype="<f4")
        out += struct.pack("<i", a.nbytes) + a.tobytes() + struct.pack("<i", a.nbytes)
    return out


def split(data):
    return [data[o:o + NMAXREC] for o in range(0, data.size, NMAXREC)]


def model_file_bytes(cubes):
    """WRITE_MODEL3D_V3 of cubes (13, NX, NY, NZ) (C order = file order)."""
    _, nx, ny, nz = cubes.shape
    data = np.ascontiguousarray(cubes, dtype=np.float32).reshape(-1)
    recs = split(data)
    head = np.array([3003, 2997, 130904, len(recs) + 1, 4, 13, nx, ny, nz], dtype=np.float32)
    return record_bytes([head] + recs)


def profile_file_bytes(ind, wave, stokes):
    """WRITE_PROFILES3D_V3 of stokes (NX, NY, NW, 4) (C order = file order)."""
    nx, ny, nw, _ = stokes.shape
    recs = split(np.ascontiguousarray(stokes, dtype=np.float32).reshape(-1))
    head = np.array([3003, 2997, 160904, len(recs) + 3, 4, nx, ny, nw, 4], dtype=np.float32)
    return record_bytes([head, np.float32(ind), np.float32(wave)] + recs)


def rf_file_bytes(z, logv, ind, wave, data):
    """WRITE_RFS3D_V3 of data (NX, NY, NZ, NW, 4, NPAR) (C order = file order)."""
    nx, ny, nz, nw, _, _ = data.shape
    recs = split(np.ascontiguousarray(data, dtype=np.float32).reshape(-1))
    head = np.array([3003, 2997, 18060904, len(recs) + 5, 6, nx, ny, nz, nw, 4, 8], dtype=np.float32)
    return record_bytes([head, np.float32(z), np.float32(ind), np.float32(wave),
                         np.float32([1.0 if v else 0.0 for v in logv])] + recs)


def model_from_cubes(cubes):
    """MODEL(NZ,13,NY*NX) as (npix, 13, nz) from cubes (13, NX, NY, NZ)."""
    _, nx, ny, nz = cubes.shape
    c = cubes.reshape(13, nx * ny, nz)
    m = np.zeros((nx * ny, 13, nz), dtype=np.float32)
    for r, k in enumerate(CUBE_OF_ROW):
        if k is None:
            continue
        m[:, r, :] = c[12, 0][None, :] if k == 12 else c[k]
    return m


def cubes_from_model(model, nx, ny, x, y):
    """WRITE_MODEL3D_V3's cubes (13, NX, NY, NZ) of model (npix, 13, nz)."""
    nz = model.shape[2]
    c = np.zeros((13, nx, ny, nz), dtype=np.float32)
    m = model.reshape(nx, ny, 13, nz)
    for k, r in enumerate(ROW_OF_CUBE):
        c[k] = m[:, :, r, :]
    c[10] = np.float32(np.asarray(x, dtype=np.float64))[:, None, None]
    c[11] = np.float32(np.asarray(y, dtype=np.float64))[None, :, None]
    c[12] = m[:, :, 12, :]
    return c


def obs_from_stokes(stokes):
    """OBS3D (npix, 4, NW) REAL*8 of STOKES (NX, NY, NW, 4)."""
    nx, ny, nw, _ = stokes.shape
    return np.transpose(stokes.reshape(nx * ny, nw, 4), (0, 2, 1)).astype(np.float64)


def stokes_from_syn(syn, nx, ny):
    """STOKES (NX, NY, NW, 4) REAL*4 of RSYN1D (npix, 4, NW)."""
    nw = syn.shape[2]
    return np.transpose(syn, (0, 2, 1)).astype(np.float32).reshape(nx, ny, nw, 4)


def rf_payload(rf_full, nx, ny):
    """DSTOKES (NX, NY, NZ, NW, 4, 6) of fz_forward_rf_full's output (npix, 6,
    NZ, 4*NW) (parameters T, Pg, Bx, By, Bz, vz)."""
    npix, six, nz, nf = rf_full.shape
    nw = nf // 4
    r = rf_full.reshape(npix, six, nz, 4, nw)
    return np.ascontiguousarray(np.transpose(r, (0, 2, 4, 3, 1))).reshape(nx, ny, nz, nw, 4, six)
