// Host-side set-up of the firtez-dz B200 library: the lines_database.dat
// reader (with the ABO collision-parameter look-up) and the Zeeman patterns.
// These run once per line set, before any kernel.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fz_host.h"
#include "fz_tables.h"
#include "fz_pftable.h"

namespace {

const double EVOLT = 1.60217656e-12;
const double HPLA = 6.62606957e-27;
const double LIGHT = 2.99792458e+10;

inline double f32(double x) { return (double)(float)x; }

std::vector<std::string> tokens(const std::string& ln) {
  std::vector<std::string> t;
  size_t i = 0;
  while (i < ln.size()) {
    while (i < ln.size() && (ln[i] == ' ' || ln[i] == '\t' || ln[i] == '\r')) ++i;
    size_t j = i;
    while (j < ln.size() && !(ln[j] == ' ' || ln[j] == '\t' || ln[j] == '\r')) ++j;
    if (j > i) t.push_back(ln.substr(i, j - i));
    i = j;
  }
  return t;
}

// Term "S.0L J.0" -> S, L, J as ELECCONF (src/lines_database.f90:692-738):
// multiplicity and J are read as REAL*4 F3.1 fields.
bool term(const std::string& e, double& S, double& L, double& J) {
  if (e.size() < 7) return false;
  static const char* ls = "SPDFGHI";
  const char* p = std::strchr(ls, e[3]);
  if (!p || !e[3]) return false;
  S = ((double)std::strtof(e.substr(0, 3).c_str(), nullptr) - 1.0) / 2.0;
  L = (double)(p - ls);
  J = (double)std::strtof(e.substr(4, 3).c_str(), nullptr);
  return true;
}

// Numeric column of the 13-column format: read as REAL*4, then rounded to
// 1e-6 (src/lines_database.f90:245-270).
double num13(const std::string& t) {
  double d = (t.find('.') != std::string::npos) ? (double)std::strtof(t.c_str(), nullptr)
                                                 : (double)(float)std::strtol(t.c_str(), nullptr, 10);
  return (double)std::llround(d * 1.0e6) * 1.0e-6;
}

// Numeric column of the 8-column format: REAL*8, rounded to 1e-4 (:347-350).
double num8(const std::string& t) { return (double)std::lround(std::strtod(t.c_str(), nullptr) * 1.e4) * 1.e-4; }

// Effective quantum numbers of the levels (GET_NEFF, src/damping.f90:1016-1090).
void neff(const fz_line& ln, double& nlow, double& nupp) {
  double xlow = ln.eplow * EVOLT;
  double xupp = xlow + HPLA * LIGHT / (ln.l0 * f32(1e-8));
  double xh = fz_tab_xii[0] * EVOLT;
  double xll, xlu;
  if (ln.elowlim != 0.0 && ln.eupplim != 0.0) {
    xll = ln.elowlim;
    xlu = ln.eupplim;
  } else {
    const double xl = (ln.ion == 1 && ln.zn > 1) ? fz_tab_xi[ln.zn - 1] * EVOLT : fz_tab_xii[ln.zn - 1] * EVOLT;
    xll = xl / (HPLA * LIGHT);
    xlu = xl / (HPLA * LIGHT);
  }
  xlow = xlow / (HPLA * LIGHT);
  xupp = xupp / (HPLA * LIGHT);
  xh = xh / (HPLA * LIGHT);
  nlow = std::sqrt(xh / (xll - xlow));
  nupp = std::sqrt(xh / (xlu - xupp));
}

// Bilinear ABO look-up on an (NX x NY) grid with origins gx0, gy0 and step
// 0.1 (REAL*4), as TRANSITION_SP/PD/DF (src/damping.f90:1126-1305).  The s-p
// table decides the lower y cell against the s grid (:1160); kept.
void abo(const double* cs, const double* al, int NX, int NY, double gx0, double gy0, double nx, double ny,
         bool sp_quirk, double& sigma, double& alpha) {
  auto gx = [&](int i) { return gx0 + (double)i * f32(0.1); };
  auto gy = [&](int i) { return gy0 + (double)i * f32(0.1); };
  int ix = 0, iy = 0;
  for (int i = 1; i < NX; ++i)
    if (std::fabs(nx - gx(i)) < std::fabs(nx - gx(ix))) ix = i;
  for (int i = 1; i < NY; ++i)
    if (std::fabs(ny - gy(i)) < std::fabs(ny - gy(iy))) iy = i;
  if (nx < gx(ix)) --ix;
  if (ny < (sp_quirk ? 1.0 + (double)iy * f32(0.1) : gy(iy))) --iy;
  ix = std::max(0, std::min(ix, NX - 2));
  iy = std::max(0, std::min(iy, NY - 2));
  const double a1 = std::fabs((gx(ix + 1) - nx) * (gy(iy + 1) - ny));
  const double a2 = std::fabs((gx(ix) - nx) * (gy(iy + 1) - ny));
  const double a3 = std::fabs((gx(ix) - nx) * (gy(iy) - ny));
  const double a4 = std::fabs((gx(ix + 1) - nx) * (gy(iy) - ny));
  const double at = a1 + a2 + a3 + a4;
  auto C = [&](const double* t, int i, int j) { return t[i * NY + j]; };
  sigma = (C(cs, ix, iy) * a1 + C(cs, ix + 1, iy) * a2 + C(cs, ix + 1, iy + 1) * a3 + C(cs, ix, iy + 1) * a4) / at;
  alpha = (C(al, ix, iy) * a1 + C(al, ix + 1, iy) * a2 + C(al, ix + 1, iy + 1) * a3 + C(al, ix, iy + 1) * a4) / at;
}

void collisional(fz_line& ln) {
  double nlow, nupp;
  neff(ln, nlow, nupp);
  const int tt = ln.otr[0] + ln.otr[1];
  double n1 = 0.0, n2 = 0.0, sig = ln.sigma, alp = ln.alpha;
  int ierr = 0;
  auto pick = [&](int o1, int o2) {   // n1 = level with orbital o1, n2 = orbital o2
    if (ln.otr[0] == o1) n1 = nlow;
    if (ln.otr[0] == o2) n2 = nlow;
    if (ln.otr[1] == o1) n1 = nupp;
    if (ln.otr[1] == o2) n2 = nupp;
  };
  if (tt == 1) {
    pick(0, 1);
    if (n1 > 5.5 || n1 < 1. || n2 > 5.5 || n2 < f32(1.3)) ierr = 3;
    if (!ierr) abo(&fz_tab_abo_cs_sp[0][0], &fz_tab_abo_al_sp[0][0], 46, 43, 1.0, f32(1.3), n1, n2, true, sig, alp);
  } else if (tt == 3) {
    pick(1, 2);
    if (n1 > 5.5 || n1 < f32(1.3) || n2 > 5.5 || n2 < f32(2.3)) ierr = 3;
    if (!ierr) abo(&fz_tab_abo_cs_pd[0][0], &fz_tab_abo_al_pd[0][0], 43, 33, f32(1.3), f32(2.3), n1, n2, false, sig, alp);
  } else if (tt == 5) {
    pick(2, 3);
    if (n1 > 5.5 || n1 < f32(2.3) || n2 > 6. || n2 < f32(3.3)) ierr = 3;
    if (!ierr) abo(&fz_tab_abo_cs_df[0][0], &fz_tab_abo_al_df[0][0], 33, 28, f32(2.3), f32(3.3), n1, n2, false, sig, alp);
  } else {
    ierr = 1;
  }
  ln.abo_ierr = ierr;
  if (!ierr) {
    ln.sigma = sig;
    ln.alpha = alp;
  }
}

}  // namespace

int fzh_lines_parse(const char* text, fz_line* out, int maxn) {
  if (!text || !out || maxn <= 0) return FZ_ERR_ARG;
  const std::string all(text);
  size_t pos = 0;
  int n = 0;
  std::string shell = "  ";   // persists across rows like the reference's local
  while (pos < all.size()) {
    size_t e = all.find('\n', pos);
    if (e == std::string::npos) e = all.size();
    const std::vector<std::string> t = tokens(all.substr(pos, e - pos));
    pos = e + 1;
    if (t.empty()) continue;
    if (t.size() == 1 && t[0] == "END") return n;
    if (n >= maxn) return FZ_ERR_LIMIT;
    fz_line L;
    std::memset(&L, 0, sizeof(L));
    if (t.size() != 13 && t.size() != 8) return FZ_ERR_PARSE;
    L.num = (int)std::strtol(t[0].c_str(), nullptr, 10);
    L.zn = (int)std::strtol(t[1].c_str(), nullptr, 10);
    L.ion = (int)std::strtol(t[2].c_str(), nullptr, 10);
    if (L.zn < 1 || L.zn > FZ_NELEM || L.ion < 1 || L.ion > 3) return FZ_ERR_PARSE;
    if (!term(t[4], L.sl, L.ll, L.jl) || !term(t[5], L.su, L.lu, L.ju)) return FZ_ERR_PARSE;
    if (t.size() == 13) {
      L.l0 = num13(t[3]);
      L.loggf = num13(t[6]);
      L.eplow = num13(t[7]);
      L.alpha = num13(t[8]);
      L.sigma = num13(t[9]);
      shell = t[10].substr(0, 2);
      L.elowlim = num13(t[11]);
      L.eupplim = num13(t[12]);
    } else {
      L.l0 = num8(t[3]);
      L.loggf = num8(t[6]);
      L.eplow = num8(t[7]);
    }
    // optical-electron transition (OPTICAL_ELEC_TRAN, src/lines_database.f90:742-787)
    for (int i = 0; i < 2; ++i) {
      const char ch = i < (int)shell.size() ? shell[i] : ' ';
      const char* orb = std::strchr("sSpPdDfF", ch);
      L.flag = 1;
      if (ch && orb) {
        L.otr[i] = (int)(orb - "sSpPdDfF") / 2;
        L.flag = 0;
      }
    }
    L.abo_ierr = -1;
    if ((L.alpha == 0.0 || L.sigma == 0.0) && L.flag == 0) collisional(L);
    out[n++] = L;
  }
  return FZ_ERR_PARSE;   // no END terminator
}

// Zeeman pattern of one line in LS coupling: ZEEMAN_COMP, src/magsplit.f90:38-187.
int fzh_zeeman(const fz_line& ln, std::vector<double>& shift, std::vector<double>& strength, std::vector<int>& type) {
  shift.clear();
  strength.clear();
  type.clear();
  const double jl = ln.jl, ju = ln.ju;
  const int dj = (int)(ju - jl);
  if (std::abs(dj) > 1) return FZ_ERR_ARG;
  const double gl = jl != 0 ? 1.5 + (ln.sl * (ln.sl + 1.0) - ln.ll * (ln.ll + 1.0)) / (2.0 * jl * (jl + 1.0)) : 0.0;
  const double gu = ju != 0 ? 1.5 + (ln.su * (ln.su + 1.0) - ln.lu * (ln.lu + 1.0)) / (2.0 * ju * (ju + 1.0)) : 0.0;
  const int nl = (int)(2 * jl + 1), nu = (int)(2 * ju + 1);
  for (int j = 0; j < nl; ++j) {
    const double ml = (double)j - jl;
    for (int k = 0; k < nu; ++k) {
      const double mu = (double)k - ju;
      const int dm = (int)(mu - ml);
      if (std::abs(dm) > 1) continue;
      double s = 0.0;
      if (dj == -1) s = dm == -1 ? (jl + mu) * (ju + mu + 2.0) : dm == 0 ? 2.0 * (jl * jl - mu * mu) : (jl - mu) * (ju - mu + 2.0);
      if (dj == 0) s = dm == -1 ? (ju - mu) * (ju + mu + 1.0) : dm == 0 ? 2.0 * mu * mu : (ju + mu) * (ju - mu + 1.0);
      if (dj == 1) s = dm == -1 ? (ju - mu) * (jl - mu) : dm == 0 ? 2.0 * (ju * ju - mu * mu) : (ju + mu) * (jl + mu);
      shift.push_back((double)(float)(4.66685e-10 * (ml * gl - mu * gu) * (ln.l0 * ln.l0)));   // mA/G, REAL*4
      strength.push_back(s);
      type.push_back(dm);
    }
  }
  double sum[3] = {0, 0, 0};
  for (size_t i = 0; i < type.size(); ++i) sum[type[i] + 1] += strength[i];
  for (size_t i = 0; i < type.size(); ++i) strength[i] /= sum[type[i] + 1];
  return (int)type.size();
}

void fzh_pf_table(PFTable* t) {
  std::memset(t, 0, sizeof(*t));
  for (int e = 0; e < FZ_NELEM; ++e)
    for (int s = 0; s < 3; ++s) {
      t->nv[e][s] = fz_tab_pf_nv[e][s];
      for (int i = 0; i < fz_tab_pf_nv[e][s]; ++i) {
        const fz_pf_vpiece& v = fz_tab_pf_v[e][s][i];
        PFPiece& p = t->p[e][s][i];
        for (int k = 0; k < v.nc && k < 6; ++k) p.c[k] = v.c[k];
        p.th = v.th;
        p.base = v.base;
        p.clamp = v.clamp;
        p.cond = v.cond;
        p.form = v.form;
        p.var = v.var;
      }
    }
}

int fzh_pfd_table(PFDTable* t) {
  std::memset(t, 0, sizeof(*t));
  for (int e = 0; e < FZ_NELEM; ++e)
    for (int s = 0; s < 3; ++s) {
      if (fz_tab_pf_nd[e][s] > 3) return -1;
      t->nd[e][s] = fz_tab_pf_nd[e][s];
      for (int i = 0; i < fz_tab_pf_nd[e][s]; ++i) {
        const fz_pf_dpiece& v = fz_tab_pf_d[e][s][i];
        if (v.nc > 6 || v.dx > 1 || v.up > 1 || v.ref > 2) return -1;
        PFDPiece& p = t->d[e][s][i];
        for (int k = 0; k < v.nc; ++k) p.c[k] = v.c[k];
        p.th = v.th;
        p.base = v.base;
        p.mult = v.mult;
        p.cond = v.cond;
        p.var = v.var;
        p.dx = v.dx;
        p.ub = v.ub;
        p.up = v.up;
        p.ref = v.ref;
      }
    }
  return 0;
}
