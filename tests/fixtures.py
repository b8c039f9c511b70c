"""Readers for the reference fixtures in tests/golden (test infrastructure)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def read_v3_model(path):
    """v3 model file (src/misc.f90:380-500) -> (ncol, 13, nz) MODEL columns."""
    from scipy.io import FortranFile
    f = FortranFile(path, "r")
    hdr = f.read_reals(np.float32)
    nx, ny, nz = int(hdr[-3]), int(hdr[-2]), int(hdr[-1])
    data = np.concatenate([f.read_reals(np.float32) for _ in range(int(hdr[3]) - 1)])
    d = data.reshape(13, nx, ny, nz)
    # file order T,Pg,rho,Bx,By,Bz,vz,Pe,mu,tau,x,y,z -> MODEL order
    order = {0: 0, 1: 1, 2: 2, 7: 3, 8: 4, 3: 5, 4: 6, 5: 7, 6: 10, 9: 11}
    m = np.zeros((nx * ny, 13, nz), dtype=np.float32)
    for src, dst in order.items():
        m[:, dst] = d[src].reshape(nx * ny, nz)
    m[:, 12] = d[12].reshape(nx * ny, nz)
    return m


def fixture_model(name="test_atmos.bin"):
    return read_v3_model(os.path.join(GOLDEN, name))


def fixture_abundances():
    return np.load(os.path.join(GOLDEN, "abund_fixture.npy"))


def fixture_lines_text():
    with open(os.path.join(GOLDEN, "lines_database.dat")) as fh:
        return fh.read()
