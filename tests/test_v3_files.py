"""v3 files on the host (CPU, no GPU): the library's C++ record I/O against
the reference's own files and writers.

* tests/golden/test_atmos.bin, rf_test_atmos.bin -- the reference's fixture
  models (default/): read, and written back byte for byte.
* v3_model_pywriter.bin, v3_profile_pywriter.bin -- files written by the
  reference's Python module (tests/golden/make_v3_golden.py): the library's
  writers reproduce them byte for byte from the same arrays.
* v3_golden.npz rf_ref_* -- what the reference's read_rf returns for the
  oracle's WRITE_RFS3D_V3 layout: the library's RF file equals the oracle's
  bytes, and its reader returns the same arrays.
* the oracle (oracle/v3_oracle.py) against the same fixtures; malformed
  files are refused with FZ_ERR_PARSE / FZ_ERR_LIMIT.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import v3_oracle as vo  # noqa: E402


@pytest.fixture(scope="module")
def v3(fz):
    from firtez_dz_b200 import v3io
    return v3io


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "v3_golden.npz"))


def _bytes(p):
    return open(p, "rb").read()


def test_oracle_matches_reference_files(gold):
    for name in ("test_atmos.bin", "rf_test_atmos.bin"):
        recs = vo.read_records(os.path.join(GOLD, name))
        nx, ny, nz = (int(v) for v in recs[0][6:9])
        assert vo.model_file_bytes(recs[1].reshape(13, nx, ny, nz)) == _bytes(os.path.join(GOLD, name))
    assert vo.model_file_bytes(gold["model_cubes"]) == _bytes(os.path.join(GOLD, "v3_model_pywriter.bin"))
    st = np.transpose(gold["prof_stokes"], (2, 3, 1, 0))
    assert (vo.profile_file_bytes(gold["prof_ind"], gold["prof_wave"], st)
            == _bytes(os.path.join(GOLD, "v3_profile_pywriter.bin")))
    q = 0
    for i, n in enumerate(("tem", "pg", "rho", "bx", "by", "bz", "vz", "p0")):
        if gold["rf_logv"][i]:
            np.testing.assert_array_equal(gold["rf_ref_" + n], gold["rf_data"][..., q])
            q += 1


@pytest.mark.parametrize("name", ["test_atmos.bin", "rf_test_atmos.bin"])
def test_reference_model_files_round_trip(v3, tmp_path, name):
    src = os.path.join(GOLD, name)
    fid, ver, dims = v3.read_header(src)
    assert (fid, ver, dims) == (130904, 3, (13, 1, 1, 256))
    cubes = v3.read_model(src)
    np.testing.assert_array_equal(cubes.reshape(-1), vo.read_records(src)[1])
    out = tmp_path / "m.bin"
    v3.write_model(out, cubes)
    assert _bytes(out) == _bytes(src)


def test_writers_match_reference_python(v3, gold, tmp_path):
    out = tmp_path / "m.bin"
    v3.write_model(out, gold["model_cubes"])
    assert _bytes(out) == _bytes(os.path.join(GOLD, "v3_model_pywriter.bin"))
    np.testing.assert_array_equal(v3.read_model(out), gold["model_cubes"])
    st = np.transpose(gold["prof_stokes"], (2, 3, 1, 0))
    out = tmp_path / "p.bin"
    v3.write_profile(out, gold["prof_ind"], gold["prof_wave"], st)
    assert _bytes(out) == _bytes(os.path.join(GOLD, "v3_profile_pywriter.bin"))
    ind, wave, st2 = v3.read_profile(out)
    np.testing.assert_array_equal(st2, st)
    np.testing.assert_array_equal(ind, np.float32(gold["prof_ind"]))
    np.testing.assert_array_equal(wave, np.float32(gold["prof_wave"]))


def test_rf_file_matches_reference_reader(v3, gold, tmp_path):
    out = tmp_path / "rf.bin"
    args = (gold["rf_z"], gold["rf_logv"], gold["rf_ind"], gold["rf_wave"], gold["rf_data"])
    v3.write_rf(out, *args)
    assert _bytes(out) == vo.rf_file_bytes(*args)
    z, logv, ind, wave, data = v3.read_rf(out)
    np.testing.assert_array_equal(logv, gold["rf_logv"])
    np.testing.assert_array_equal(z, np.float32(gold["rf_z"]))
    q = 0
    for i, n in enumerate(("tem", "pg", "rho", "bx", "by", "bz", "vz", "p0")):
        if logv[i]:
            np.testing.assert_array_equal(data[..., q], gold["rf_ref_" + n])
            q += 1


def test_malformed_files_refused(fz, v3, gold, tmp_path):
    src = _bytes(os.path.join(GOLD, "v3_model_pywriter.bin"))
    # a profile file is not a model file
    with pytest.raises(fz.FzError):
        v3.read_model(os.path.join(GOLD, "v3_profile_pywriter.bin"))
    # truncated payload
    bad = tmp_path / "trunc.bin"
    bad.write_bytes(src[:-20])
    with pytest.raises(fz.FzError):
        v3.read_model(bad)
    # damaged trailing record marker
    bad.write_bytes(src[:-1] + b"\x7f")
    with pytest.raises(fz.FzError):
        v3.read_model(bad)
    # version 2 header
    b = bytearray(src)
    b[4:12] = np.array([3002, 2998], dtype="<f4").tobytes()
    bad.write_bytes(bytes(b))
    with pytest.raises(fz.FzError):
        v3.read_model(bad)
    # dimensions differ from the caller's
    good = tmp_path / "m.bin"
    v3.write_model(good, gold["model_cubes"])
    buf = np.empty(13 * 4 * 2 * 4, dtype=np.float32)
    rc = fz.lib().fz_v3_read_model(str(good).encode(), 4, 2, 4, buf.ctypes.data_as(__import__("ctypes").c_void_p))
    assert rc == -5   # FZ_ERR_LIMIT
    # a missing file
    with pytest.raises(fz.FzError):
        v3.read_header(tmp_path / "none.bin")


def test_lsf_file_matches_reference_writer(v3, gold, tmp_path):
    """The LSF file (READ_LSF_FILE's format) byte for byte as the reference's
    Python write_lsf writes it, and read back."""
    out = tmp_path / "lsf.bin"
    v3.write_lsf(out, gold["lsf"])
    assert _bytes(out) == _bytes(os.path.join(GOLD, "v3_lsf_pywriter.bin"))
    np.testing.assert_array_equal(v3.read_lsf(out, gold["lsf"].size), np.float32(gold["lsf"]).astype(np.float64))
    with pytest.raises(Exception):
        v3.read_lsf(out, gold["lsf"].size + 1)


def test_multi_record_model_file(v3, tmp_path):
    """A model above NMAXREC = 268,435,446 values (13 x 4096 x 5042, 1.07 GB)
    goes into two data records, as WRITE_MODEL3D_V3 splits it: the header's
    record count, both records' markers and sizes, and the read-back."""
    import struct
    nx, ny, nz = 64, 64, 5042
    n = 13 * nx * ny * nz
    assert n > vo.NMAXREC
    cubes = np.zeros((13, nx, ny, nz), dtype=np.float32)
    cubes.reshape(-1)[::9973] = np.arange(cubes.size // 9973 + 1, dtype=np.float32)[: cubes.reshape(-1)[::9973].size]
    out = tmp_path / "big.bin"
    v3.write_model(out, cubes)
    with open(out, "rb") as f:
        assert struct.unpack("<i", f.read(4))[0] == 36
        head = np.frombuffer(f.read(36), "<f4")
        assert head[3] == 3 and struct.unpack("<i", f.read(4))[0] == 36     # header + 2 data records
        for size in (vo.NMAXREC, n - vo.NMAXREC):
            b0 = struct.unpack("<i", f.read(4))[0]
            f.seek(b0, 1)
            assert b0 == 4 * size and struct.unpack("<i", f.read(4))[0] == b0
        assert f.read(1) == b""
    back = v3.read_model(out)
    out.unlink()
    assert np.array_equal(back, cubes)
