#!/usr/bin/env python3
"""Copy the reference's data fixtures into tests/golden/ and extract the
alternative abundance set they were generated with.

TEST INFRASTRUCTURE.  Reads the reference tree given as the one argument:

  default/test_atmos.bin, default/rf_test_atmos.bin  -- v3 model files (1x1x256)
  default/lines_database.dat                         -- line database
  tests/*/control_file.dat                           -- the test cases' control
      files (copied to control/<case>.dat)
  src/atom_database.f90:89-97                         -- the commented-out
      "Abundances Vigeesh" set; the fixtures' rho, Pe, mu were computed with it.
"""
import os
import re
import shutil
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_fixtures.py <path of the reference tree>")
ref = sys.argv[1]
here = os.path.dirname(os.path.abspath(__file__))
for f in ("test_atmos.bin", "rf_test_atmos.bin", "lines_database.dat"):
    shutil.copyfile(os.path.join(ref, "default", f), os.path.join(here, f))
os.makedirs(os.path.join(here, "control"), exist_ok=True)
for case in sorted(os.listdir(os.path.join(ref, "tests"))):
    cf = os.path.join(ref, "tests", case, "control_file.dat")
    if os.path.isfile(cf):
        shutil.copyfile(cf, os.path.join(here, "control", case + ".dat"))
src = open(os.path.join(ref, "src", "atom_database.f90")).read().splitlines()
i0 = next(i for i, l in enumerate(src) if "Abundances Vigeesh" in l)
txt = ""
for l in src[i0 + 1:]:
    l = l.lstrip()
    if not l.startswith("!"):
        break
    txt += l.lstrip("!").strip().rstrip("&")
body = txt[txt.index("(/") + 2:txt.index("/)")]
ab = np.array([float(np.float32(float(x))) for x in body.replace("&", "").split(",") if x.strip()])
assert len(ab) == 92, len(ab)
np.save(os.path.join(here, "abund_fixture.npy"), ab)
print("fixtures written to", here)
