"""The C-ABI library on the CPU side: it loads without a GPU, exports every
symbol of include/fz_b200.h, and its line-database reader (host code) equals
the oracle's restatement of NREAD_LINES_DATABASE on the reference database."""
import os
import re

import numpy as np

import fixtures

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(fz_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol(fz):
    L = fz.lib()
    names = declared_symbols()
    assert "fz_forward" in names and "fz_create" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_line_parser_matches_oracle(fz, orc):
    text = fixtures.fixture_lines_text()
    a = fz.lines_parse(text)
    b = orc.parse_lines(text)
    assert len(a) == len(b) == 37
    for f in fz.LINE_DTYPE.names:
        if f == "pad":
            continue
        assert np.array_equal(a[f], b[f]), f
    fe = a[a["num"] == 4][0]
    assert fe["flag"] == 0 and fe["abo_ierr"] == 0 and fe["sigma"] > 0 and fe["alpha"] > 0
    assert fe["l0"] == 6301.500977            # REAL*4 read, rounded to 1e-6


def test_line_parser_workload_database(fz, orc):
    text = fz.atmos.line_database_text()
    a, b = fz.lines_parse(text), orc.parse_lines(text)
    for f in ("l0", "loggf", "eplow", "alpha", "sigma", "sl", "ll", "jl", "su", "lu", "ju"):
        assert np.array_equal(a[f], b[f]), f


def test_parser_rejects_malformed(fz):
    import pytest
    with pytest.raises(fz.FzError):
        fz.lines_parse("1 026 1 6301.5 5.0P2.0\nEND\n")
    with pytest.raises(fz.FzError):
        fz.lines_parse("1  026  1   6301.5010  5.0P2.0  5.0D2.0  -0.720  3.654  0.000  0000.000 ps 0 0\n")


def test_regions_from_lines_section(fz):
    lines = fz.lines_parse(fixtures.fixture_lines_text())
    reg = fz.regions_from_lines_section("4,5 500 -700.0 5.0", lines)
    assert reg["nblend"][0] == 2 and reg["numwave"][0] == 500
    assert abs(reg["wdif"][0, 1] - 1e3 * (6302.493652 - 6301.500977)) < 1e-6


def _c_layout(tmp_path, struct, fields):
    """sizeof and offsetof of a C struct of include/fz_b200.h (gcc)."""
    import subprocess
    src = tmp_path / ("probe_%s.c" % struct)
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fz_b200.h"', "int main(void) {",
             '  printf("%%zu\\n", sizeof(%s));' % struct]
    lines += ['  printf("%%zu\\n", offsetof(%s, %s));' % (struct, f) for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / ("probe_%s" % struct)
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    return out[0], dict(zip(fields, out[1:]))


def test_struct_layouts_match_the_header(fz, tmp_path):
    """The ctypes / numpy mirrors of fz_lm_opts, fz_tune, fz_line and
    fz_region have the C header's sizes and field offsets."""
    import ctypes
    for struct, cls in (("fz_lm_opts", fz.LMOpts), ("fz_tune", fz.Tune)):
        names = [f[0] for f in cls._fields_]
        size, offs = _c_layout(tmp_path, struct, names)
        assert ctypes.sizeof(cls) == size, struct
        for n in names:
            assert getattr(cls, n).offset == offs[n], (struct, n)
    for struct, dt in (("fz_line", fz.LINE_DTYPE), ("fz_region", fz.REGION_DTYPE)):
        names = list(dt.names)
        size, offs = _c_layout(tmp_path, struct, names)
        assert dt.itemsize == size, struct
        for n in names:
            assert dt.fields[n][1] == offs[n], (struct, n)


def test_fortran_interfaces_match_the_header():
    """include/fz_b200.f90, the ISO_C_BINDING module the Fortran host uses,
    binds every function the C header declares, once, with the same number
    of arguments, and its BIND(C) types carry the C structs' fields in order.
    (gfortran is not on this image, so the module is checked as text.)"""
    hdr = "".join(open(os.path.join(ROOT, "include", f)).read()
                  for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h"))
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(fz_\w+)\s*\(([^)]*)\)\s*;", hdr):
        args = m.group(2).strip()
        protos[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    f90 = open(os.path.join(ROOT, "include", "fz_b200.f90")).read()
    f90 = re.sub(r"!.*", "", f90).replace("&\n", " ")
    found = re.findall(r"FUNCTION\s+(FZ_\w+)\(([^)]*)\)\s*BIND\(C,\s*NAME='(fz_\w+)'\)", f90)
    names = [n for _, _, n in found]
    assert sorted(names) == sorted(protos), set(names) ^ set(protos)
    for fname, args, name in found:
        assert fname == name.upper(), name
        n = 0 if not args.strip() else args.count(",") + 1
        assert n == protos[name], (name, n, protos[name])
        # every dummy argument has a declaration in the interface body
        body = f90[f90.index("NAME='%s')" % name):]
        body = body[:body.index("END FUNCTION")]
        for a in (x.strip() for x in args.split(",") if x.strip()):
            assert re.search(r"::\s*(?:[\w(),*]+\s*,\s*)*%s\b" % a, body), (name, a)
    # the BIND(C) derived types list the C structs' fields in order
    for ctype, ftype in (("fz_lm_opts", "FZ_LM_OPTS"), ("fz_tune", "FZ_TUNE"), ("fz_line", "FZ_LINE"),
                         ("fz_region", "FZ_REGION")):
        cb = re.search(r"typedef struct\s*\{([^}]*)\}\s*%s;" % ctype, hdr).group(1)
        cf = []
        for decl in cb.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            # one declaration: the type, then the comma-separated field names
            parts = decl.split(",")
            first = re.sub(r"\[.*?\]", "", parts[0]).split()[-1].lstrip("*")
            cf.append(first)
            cf += [re.sub(r"\[.*?\]", "", x).strip().lstrip("*") for x in parts[1:]]
        fb = re.search(r"TYPE, BIND\(C\) :: %s(.*?)END TYPE" % ftype, f90, flags=re.S).group(1)
        ff = []
        for ln in fb.splitlines():
            if "::" in ln:
                ff += [re.sub(r"\(.*?\)", "", x).strip() for x in ln.split("::")[1].split(",")]
        assert [x.upper() for x in cf] == ff, (ctype, cf, ff)
