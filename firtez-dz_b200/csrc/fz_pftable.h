// Compact partition-function table shared by the host builder and the
// kernels: per (element, stage) up to FZ_PF_MAXV value pieces of
// src/atom_database.f90:121-1035 with 6 (zero-padded) Horner coefficients.
#pragma once
#ifndef FZ_PF_MAXV
#define FZ_PF_MAXV 3
#endif
#ifndef FZ_NELEM
#define FZ_NELEM 92
#endif

struct PFPiece {
  double c[6];
  double th, base, clamp;
  int cond, form, var, pad;
};
struct PFTable {
  PFPiece p[FZ_NELEM][3][FZ_PF_MAXV];
  int nv[FZ_NELEM][3];
};

// Fill t from the generated piece table (host).
void fzh_pf_table(PFTable* t);
