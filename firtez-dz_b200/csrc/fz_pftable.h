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

// Derivative pieces (dlnU/dT) of src/atom_database.f90:121-1035 in the same
// padded form: the active piece is the last whose condition holds (on T, or
// on the value of the referenced value piece, ref < 0 = the stage's U);
// d = horner(c, var) * mult * (dx ? -1/T : 1) * (ub ? uref - base : 1) / (up ? uref : 1).
struct PFDPiece {
  double c[6];
  double th, base, mult;
  int cond, var, dx, ub, up, ref, pad0, pad1;
};
struct PFDTable {
  PFDPiece d[FZ_NELEM][3][3];
  int nd[FZ_NELEM][3];
};

// Fill t from the generated piece table (host).
void fzh_pf_table(PFTable* t);
// Fill t from the generated derivative pieces (host); returns 0, or -1 if a
// piece needs more than the padded form holds.
int fzh_pfd_table(PFDTable* t);
