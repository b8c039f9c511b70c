// FIRTEZ-dz v3 files on the host: the model atmosphere, Stokes profile and
// response-function files of src/misc.f90 (READ_MODEL_3D :78-503,
// WRITE_MODEL3D_V3 :801-929, WRITE_PROFILES3D_V3 :1147-1249,
// READ_PROFILE_3D :1338-1642, WRITE_RFS3D_V3 :1862-1999).
//
// A v3 file is a Fortran unformatted sequential file: records framed by a
// 4-byte little-endian byte count before and after, all payloads REAL*4.
// Record 1 is the header (POSV = 3000 + v, NEGV = 3000 - v, the file ID,
// the record count, the number of dimensions, the dimensions); the data
// follow in records of at most NMAXREC = 268,435,446 values (misc.f90:16-17;
// the reference's Python writer uses the same bound).  These routines move
// the payload as it lies in the file -- the layout changes to the device's
// MODEL(NZ,13,npix), OBS3D(NFREQ,npix) and RF arrays are GPU kernels.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>

#include "../../include/fz_b200.h"

namespace {

const int64_t kMaxRec = 1073741784 / 4;   // NMAXREC, values per data record

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) std::fclose(f);
  }
};

bool put_rec(FILE* f, const float* p, int64_t n) {
  if (n < 0 || n * 4 > 0x7fffffffLL) return false;
  const uint32_t b = (uint32_t)(n * 4);
  if (std::fwrite(&b, 4, 1, f) != 1) return false;
  if (n > 0 && std::fwrite(p, 4, (size_t)n, f) != (size_t)n) return false;
  return std::fwrite(&b, 4, 1, f) == 1;
}

// the payload of the next record into p (exactly n values expected)
bool get_rec(FILE* f, float* p, int64_t n) {
  uint32_t b0 = 0, b1 = 0;
  if (std::fread(&b0, 4, 1, f) != 1) return false;
  if ((int64_t)b0 != n * 4) return false;
  if (n > 0 && std::fread(p, 4, (size_t)n, f) != (size_t)n) return false;
  if (std::fread(&b1, 4, 1, f) != 1) return false;
  return b1 == b0;
}

// the byte count of the next record, the file position kept
bool peek_len(FILE* f, uint32_t& b) {
  const long at = std::ftell(f);
  const bool ok = std::fread(&b, 4, 1, f) == 1;
  std::fseek(f, at, SEEK_SET);
  return ok;
}

bool put_data(FILE* f, const float* p, int64_t n) {
  for (int64_t o = 0; o < n; o += kMaxRec)
    if (!put_rec(f, p + o, std::min(kMaxRec, n - o))) return false;
  return true;
}

bool get_data(FILE* f, float* p, int64_t n) {
  for (int64_t o = 0; o < n; o += kMaxRec)
    if (!get_rec(f, p + o, std::min(kMaxRec, n - o))) return false;
  return true;
}

int64_t nrec_data(int64_t n) { return (n + kMaxRec - 1) / kMaxRec; }

// Header record: version from (POSV - NEGV) / 2 with MEDV = 3000 (READ_MODEL,
// misc.f90:507-553), the ID, record count, dimension count and sizes.
int read_header(FILE* f, float* h, int& nh) {
  uint32_t b = 0;
  if (!peek_len(f, b) || b % 4 || b < 20 || b > 64) return FZ_ERR_PARSE;
  nh = (int)(b / 4);
  if (!get_rec(f, h, nh)) return FZ_ERR_PARSE;
  const int posv = (int)h[0], negv = (int)h[1];
  if ((posv + negv) / 2 != 3000 || posv + negv != 6000) return FZ_ERR_PARSE;
  return 0;
}

int check_open(File& F, const char* path, const char* mode) {
  if (!path) return FZ_ERR_ARG;
  F.f = std::fopen(path, mode);
  return F.f ? 0 : FZ_ERR_ARG;
}

}  // namespace

extern "C" {

int fz_v3_header(const char* path, int* id, int* version, int* ndims, int dims[8]) {
  File F;
  if (int rc = check_open(F, path, "rb")) return rc;
  float h[16] = {0};
  int nh = 0;
  if (int rc = read_header(F.f, h, nh)) return rc;
  const int nd = (int)h[4];
  if (nd < 0 || nd > 8 || 5 + nd > nh) return FZ_ERR_PARSE;
  if (id) *id = (int)h[2];
  if (version) *version = ((int)h[0] - (int)h[1]) / 2;
  if (ndims) *ndims = nd;
  if (dims)
    for (int i = 0; i < 8; ++i) dims[i] = i < nd ? (int)h[5 + i] : 0;
  return 0;
}

int fz_v3_read_model(const char* path, int nx, int ny, int nz, float* cubes) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !cubes) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "rb")) return rc;
  float h[16];
  int nh = 0;
  if (int rc = read_header(F.f, h, nh)) return rc;
  // READ_MODEL_3D version 3 (misc.f90:374-499): ID 130904, 4 dimensions,
  // NPAR = 13 and the grid of the caller
  if (nh != 9 || std::fabs(h[2] - 130904.f) > 0.01f || (int)h[0] - (int)h[1] != 6 || (int)h[4] != 4)
    return FZ_ERR_PARSE;
  if ((int)h[5] != 13 || (int)h[6] != nx || (int)h[7] != ny || (int)h[8] != nz) return FZ_ERR_LIMIT;
  const int64_t n = 13LL * nx * ny * nz;
  if ((int64_t)h[3] != 1 + nrec_data(n)) return FZ_ERR_PARSE;
  return get_data(F.f, cubes, n) ? 0 : FZ_ERR_PARSE;
}

int fz_v3_write_model(const char* path, int nx, int ny, int nz, const float* cubes) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !cubes) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "wb")) return rc;
  const int64_t n = 13LL * nx * ny * nz;
  // WRITE_MODEL3D_V3 (misc.f90:801-929)
  const float h[9] = {3003.f, 2997.f, 130904.f, (float)(1 + nrec_data(n)), 4.f, 13.f, (float)nx, (float)ny,
                      (float)nz};
  if (!put_rec(F.f, h, 9) || !put_data(F.f, cubes, n)) return FZ_ERR_ARG;
  return std::fclose(std::exchange(F.f, nullptr)) == 0 ? 0 : FZ_ERR_ARG;
}

int fz_v3_read_profiles(const char* path, int nx, int ny, int nw, float* ind, float* wave, float* stokes) {
  if (nx <= 0 || ny <= 0 || nw <= 0 || !stokes) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "rb")) return rc;
  float h[16];
  int nh = 0;
  if (int rc = read_header(F.f, h, nh)) return rc;
  // READ_PROFILE_3D version 3: ID 160904, dims (NX, NY, NW, 4)
  if (nh != 9 || std::fabs(h[2] - 160904.f) > 0.01f || (int)h[0] - (int)h[1] != 6 || (int)h[4] != 4)
    return FZ_ERR_PARSE;
  if ((int)h[5] != nx || (int)h[6] != ny || (int)h[7] != nw || (int)h[8] != 4) return FZ_ERR_LIMIT;
  const int64_t n = 4LL * nw * ny * nx;
  if ((int64_t)h[3] != 3 + nrec_data(n)) return FZ_ERR_PARSE;
  std::vector<float> tmp;
  if (!ind || !wave) tmp.resize(nw);
  if (!get_rec(F.f, ind ? ind : tmp.data(), nw) || !get_rec(F.f, wave ? wave : tmp.data(), nw)) return FZ_ERR_PARSE;
  return get_data(F.f, stokes, n) ? 0 : FZ_ERR_PARSE;
}

int fz_v3_write_profiles(const char* path, int nx, int ny, int nw, const double* ind, const double* wave,
                         const float* stokes) {
  if (nx <= 0 || ny <= 0 || nw <= 0 || !ind || !wave || !stokes) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "wb")) return rc;
  const int64_t n = 4LL * nw * ny * nx;
  // WRITE_PROFILES3D_V3 (misc.f90:1147-1249): IND and WAVE as REAL(.)
  const float h[9] = {3003.f, 2997.f, 160904.f, (float)(3 + nrec_data(n)), 4.f, (float)nx, (float)ny, (float)nw,
                      4.f};
  std::vector<float> a(nw), b(nw);
  for (int i = 0; i < nw; ++i) {
    a[i] = (float)ind[i];
    b[i] = (float)wave[i];
  }
  if (!put_rec(F.f, h, 9) || !put_rec(F.f, a.data(), nw) || !put_rec(F.f, b.data(), nw) || !put_data(F.f, stokes, n))
    return FZ_ERR_ARG;
  return std::fclose(std::exchange(F.f, nullptr)) == 0 ? 0 : FZ_ERR_ARG;
}

int fz_v3_write_rfs(const char* path, int nx, int ny, int nz, int nw, const double* z, const int* logv,
                    const double* ind, const double* wave, const float* data) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || nw <= 0 || !z || !logv || !ind || !wave || !data) return FZ_ERR_ARG;
  int np = 0;
  float lv[8];
  for (int p = 0; p < 8; ++p) {
    lv[p] = logv[p] ? 1.f : 0.f;
    np += logv[p] != 0;
  }
  if (np == 0) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "wb")) return rc;
  const int64_t n = (int64_t)np * 4 * nw * nz * ny * nx;
  // WRITE_RFS3D_V3 (misc.f90:1862-1999): header of 11, then Z, IND, WAVE,
  // LOGV, then the derivatives with the parameter index fastest
  const float h[11] = {3003.f, 2997.f, 18060904.f, (float)(5 + nrec_data(n)), 6.f, (float)nx, (float)ny, (float)nz,
                       (float)nw, 4.f, 8.f};
  std::vector<float> zz(nz), a(nw), b(nw);
  for (int k = 0; k < nz; ++k) zz[k] = (float)z[k];
  for (int i = 0; i < nw; ++i) {
    a[i] = (float)ind[i];
    b[i] = (float)wave[i];
  }
  if (!put_rec(F.f, h, 11) || !put_rec(F.f, zz.data(), nz) || !put_rec(F.f, a.data(), nw) ||
      !put_rec(F.f, b.data(), nw) || !put_rec(F.f, lv, 8) || !put_data(F.f, data, n))
    return FZ_ERR_ARG;
  return std::fclose(std::exchange(F.f, nullptr)) == 0 ? 0 : FZ_ERR_ARG;
}

int fz_v3_read_rfs(const char* path, int nx, int ny, int nz, int nw, float* z, int* logv, float* ind, float* wave,
                   float* data) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || nw <= 0 || !logv) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "rb")) return rc;
  float h[16];
  int nh = 0;
  if (int rc = read_header(F.f, h, nh)) return rc;
  if (nh != 11 || std::fabs(h[2] - 18060904.f) > 1.f || (int)h[0] - (int)h[1] != 6 || (int)h[4] != 6)
    return FZ_ERR_PARSE;
  if ((int)h[5] != nx || (int)h[6] != ny || (int)h[7] != nz || (int)h[8] != nw || (int)h[9] != 4 || (int)h[10] != 8)
    return FZ_ERR_LIMIT;
  std::vector<float> tz(nz), tw(nw);
  float lv[8];
  if (!get_rec(F.f, z ? z : tz.data(), nz) || !get_rec(F.f, ind ? ind : tw.data(), nw) ||
      !get_rec(F.f, wave ? wave : tw.data(), nw) || !get_rec(F.f, lv, 8))
    return FZ_ERR_PARSE;
  int np = 0;
  for (int p = 0; p < 8; ++p) {
    logv[p] = lv[p] != 0.f;
    np += logv[p];
  }
  const int64_t n = (int64_t)np * 4 * nw * nz * ny * nx;
  if ((int64_t)h[3] != 5 + nrec_data(n)) return FZ_ERR_PARSE;
  if (!data) return np;   // the parameter count: size the data buffer, call again
  return get_data(F.f, data, n) ? np : FZ_ERR_PARSE;
}

int fz_v3_read_lsf(const char* path, int n, double* yk) {
  if (n <= 0 || !yk) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "rb")) return rc;
  float h[16];
  int nh = 0;
  if (int rc = read_header(F.f, h, nh)) return rc;
  // READ_LSF_FILE (misc.f90:2422-2555): ID 3330904, one dimension NIW
  if (nh != 6 || std::fabs(h[2] - 3330904.f) > 0.5f || (int)h[4] != 1) return FZ_ERR_PARSE;
  if ((int)h[5] != n) return FZ_ERR_LIMIT;
  std::vector<float> v(n);
  for (int64_t o = 0; o < n; o += kMaxRec)
    if (!get_rec(F.f, v.data() + o, std::min<int64_t>(kMaxRec, n - o))) return FZ_ERR_PARSE;
  for (int i = 0; i < n; ++i) yk[i] = (double)v[i];
  return 0;
}

int fz_v3_write_lsf(const char* path, int n, const double* yk) {
  if (n <= 0 || !yk) return FZ_ERR_ARG;
  File F;
  if (int rc = check_open(F, path, "wb")) return rc;
  // the reference's Python write_lsf: header 3003, 2997, 3330904, NRECS+1,
  // 1, NW (its record count is sized for 4 NW values: one record up to
  // 67,108,861 wavelengths)
  const int64_t nrec = (4 * (int64_t)n + kMaxRec - 1) / kMaxRec;
  const float h[6] = {3003.f, 2997.f, 3330904.f, (float)(nrec + 1), 1.f, (float)n};
  std::vector<float> v(n);
  for (int i = 0; i < n; ++i) v[i] = (float)yk[i];
  if (!put_rec(F.f, h, 6) || !put_data(F.f, v.data(), n)) return FZ_ERR_ARG;
  return std::fclose(std::exchange(F.f, nullptr)) == 0 ? 0 : FZ_ERR_ARG;
}

}  // extern "C"
