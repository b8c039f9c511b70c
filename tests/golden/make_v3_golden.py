#!/usr/bin/env python3
"""Golden v3 files written and read by the reference's own Python module.

TEST INFRASTRUCTURE.  Imports python/firtez_dz.py from the reference tree
(its path the one argument) with two shims that touch nothing of its file
code: a do-nothing matplotlib (the module sets up plotting at import; the
package is not installed here) and np.int = int (removed in numpy 2; the
writers use it for the record size).  Writes, next to this script:

  v3_model_pywriter.bin    atm_model3D.write (write_model3D_v3) of a seeded
                           3 x 2 x 4 model
  v3_profile_pywriter.bin  stk_profile3D.write (write_profile3D_v3) of seeded
                           3 x 2 profiles of 5 wavelengths
  v3_lsf_pywriter.bin      write_lsf of a seeded 7-point line spread function
  v3_golden.npz            the seeded inputs, and what the reference's
                           read_rf returns for a 2 x 3 x 4 x 5 RF file laid
                           out by the oracle's WRITE_RFS3D_V3 restatement
                           (oracle/v3_oracle.py)

The model and profile files pin the byte layout the library's writers must
reproduce; the RF arrays pin the RF layout through the reference's reader.
"""
import os
import sys
import tempfile
import types

import numpy as np

here = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) != 2:
    sys.exit("usage: make_v3_golden.py <path of the reference tree>")
ref = sys.argv[1]
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(here)), "oracle"))
import v3_oracle  # noqa: E402


class _Any:
    def __getattr__(self, name):
        return _Any()

    def __call__(self, *a, **k):
        return _Any()


mpl = types.ModuleType("matplotlib")
mpl.pyplot = _Any()
mpl.ticker = _Any()
mpl.rcParams = {}
sys.modules["matplotlib"] = mpl
sys.modules["matplotlib.pyplot"] = mpl.pyplot
sys.modules["matplotlib.ticker"] = mpl.ticker
mpl.pyplot.rcParams = {}
if not hasattr(np, "int"):
    np.int = int
sys.path.insert(0, os.path.join(ref, "python"))
import firtez_dz as fzpy  # noqa: E402

rng = np.random.default_rng(2024)

# ---- model (full=True: all 13 cubes)
nx, ny, nz = 3, 2, 4
cubes = rng.standard_normal((13, nx, ny, nz)).astype(np.float32) * np.float32(1000.0)
m = fzpy.atm_model3D(nx, ny, nz, full=True)
for k, name in enumerate(("tem", "pg", "rho", "bx", "by", "bz", "vz", "pel", "mw", "tau", "x", "y", "z")):
    setattr(m, name, cubes[k].astype(np.float64))
m.write(os.path.join(here, "v3_model_pywriter.bin"))

# ---- profiles
pnx, pny, nw = 3, 2, 5
stokes = rng.standard_normal((4, nw, pnx, pny)).astype(np.float32)
ind = np.arange(1, nw + 1, dtype=np.float64)
wave = (-1193.25 + 21.5 * np.arange(nw)).astype(np.float64)
p = fzpy.stk_profile3D(nw, pnx, pny)
p.set_profiles(stokes.astype(np.float64), ind, wave)
p.write(os.path.join(here, "v3_profile_pywriter.bin"))

# ---- line spread function file
lsf = rng.random(7)
lsf = lsf / lsf.sum()
fzpy.write_lsf(os.path.join(here, "v3_lsf_pywriter.bin"), lsf)

# ---- RFs: the oracle's file layout read back by the reference's reader
rnx, rny, rnz, rnw = 2, 3, 4, 5
logv = [1, 1, 0, 1, 1, 1, 1, 0]
rfdata = rng.standard_normal((rnx, rny, rnz, rnw, 4, 6)).astype(np.float32)
rz = np.linspace(0.0, 300.0, rnz)
rind = np.ones(rnw)
rwave = np.arange(rnw, dtype=np.float64)
with tempfile.TemporaryDirectory() as td:
    fn = os.path.join(td, "rf.bin")
    open(fn, "wb").write(v3_oracle.rf_file_bytes(rz, logv, rind, rwave, rfdata))
    r = fzpy.read_rf(fn)
    rf_ref = {n: np.array(getattr(r, "rf_" + n), dtype=np.float32)
              for n in ("tem", "pg", "rho", "bx", "by", "bz", "vz", "p0")}

np.savez(os.path.join(here, "v3_golden.npz"), model_cubes=cubes, prof_stokes=stokes, prof_ind=ind, prof_wave=wave,
         lsf=lsf, rf_data=rfdata, rf_z=rz, rf_ind=rind, rf_wave=rwave, rf_logv=np.array(logv, dtype=np.int32),
         **{"rf_ref_" + k: v for k, v in rf_ref.items()})
print("wrote v3_model_pywriter.bin, v3_profile_pywriter.bin, v3_lsf_pywriter.bin, v3_golden.npz")
