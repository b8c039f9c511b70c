#!/usr/bin/env python3
"""A second, independent read of the reference's data tables, as pins for
the library's generated tables.

TEST INFRASTRUCTURE.  Usage: make_table_pins.py <path of the reference tree>.
Writes table_pins.npz next to this script with

  abo_cs_sp, abo_al_sp (46, 43)  src/damping.f90 CS_SP, AL_SP
  abo_cs_pd, abo_al_pd (43, 33)  CS_PD, AL_PD
  abo_cs_df, abo_al_df (33, 28)  CS_DF, AL_DF
  hsra_tem, hsra_pg, hsra_rho, hsra_z (387)
                                 src/normalization.f90, the assignments of
                                 SUBROUTINE SET_HSRA_MODEL

It shares no code with oracle/gen_tables.py (which writes the library's
fz_tables.h): the Fortran text is flattened (comments and continuation
marks removed) and each array constructor is split on commas; element (i, j)
of a RESHAPE comes from the SOURCE list in Fortran's order, first index
fastest, or second index fastest with ORDER=(/2,1/).  A real literal without
a D exponent is a default (REAL*4) constant and is rounded to float32 before
it widens to the REAL(DP) parameter, as the compiler does.
"""
import os
import re
import sys

import numpy as np


def flatten(text):
    lines = []
    for ln in text.splitlines():
        ln = ln.split("!", 1)[0]
        lines.append(ln.rstrip())
    flat = " ".join(lines)
    return re.sub(r"&\s*&?", " ", flat)


def literal(tok):
    tok = tok.strip()
    if re.fullmatch(r"[+-]?\d+", tok):
        return float(int(tok))
    if re.search(r"[dD]", tok):
        return float(tok.replace("d", "e").replace("D", "e"))
    return float(np.float32(float(tok)))


def constructor(flat, start):
    """The comma-separated items of the (/ ... /) constructor opening at or
    after index start."""
    i = flat.index("(/", start)
    j = flat.index("/)", i)
    return [literal(t) for t in flat[i + 2:j].split(",")], j


def reshape_param(flat, name):
    m = re.search(r"\b%s\s*\(\s*(\d+)\s*,\s*(\d+)\s*\)\s*=\s*RESHAPE\s*\(" % name, flat, flags=re.I)
    n1, n2 = int(m.group(1)), int(m.group(2))
    src_at = flat.upper().index("SOURCE", m.end())
    vals, end = constructor(flat, src_at)
    tail = flat[end:end + 60].replace(" ", "").upper()
    order21 = tail.startswith("/),ORDER=(/2,1/)")
    assert len(vals) == n1 * n2, (name, len(vals))
    a = np.array(vals)
    return a.reshape(n1, n2) if order21 else a.reshape(n2, n1).T


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_table_pins.py <path of the reference tree>")
    src = os.path.join(sys.argv[1], "src")
    damp = flatten(open(os.path.join(src, "damping.f90")).read())
    out = {}
    for nm in ("CS_SP", "AL_SP", "CS_PD", "AL_PD", "CS_DF", "AL_DF"):
        out["abo_" + nm.lower()] = reshape_param(damp, nm)
    norm = flatten(open(os.path.join(src, "normalization.f90")).read())
    sub = re.search(r"SUBROUTINE\s+SET_HSRA_MODEL\b(.*?)END\s+SUBROUTINE\s+SET_HSRA_MODEL", norm, flags=re.I | re.S)
    body = sub.group(1)
    for nm in ("TEM", "PG", "RHO", "Z"):
        m = re.search(r"\bHSRA_%s\s*\(\s*:\s*\)\s*=" % nm, body)
        vals, _ = constructor(body, m.end())
        out["hsra_" + nm.lower()] = np.array(vals, dtype=np.float32)
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "table_pins.npz"), **out)
    for k, v in out.items():
        print(k, v.shape)


if __name__ == "__main__":
    main()
