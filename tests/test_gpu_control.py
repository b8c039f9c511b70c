"""The reference's own test cases run through the control-file host
(firtez-dz_b200/control.py) on the GPU, in a copy of the reference's
layout (tests/<case>/control_file.dat, default/ with the fixture model files
and line database): test_syn1 (synthesis of test_atmos.bin, 500 wavelengths
of Fe I 6301.5 blended with 6302.5, 256 heights), test_rf (with the
response functions to T and Bz at every height), test_he (hydrostatic
equilibrium only) and test_tau1 (log tau5).  The files written equal the
library's direct calls on the same model.  test_inv1 (NP = 512) runs in
tests/test_gpu_lm_big.py."""
import os
import shutil
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import v3_oracle as vo  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture()
def tree(tmp_path):
    d = tmp_path / "default"
    d.mkdir()
    for f in ("test_atmos.bin", "rf_test_atmos.bin", "lines_database.dat"):
        shutil.copyfile(os.path.join(GOLD, f), d / f)
    for case in ("test_syn1", "test_rf", "test_he", "test_tau1", "test_inv1"):
        t = tmp_path / "tests" / case
        (t / "out_dir").mkdir(parents=True)
        shutil.copyfile(os.path.join(GOLD, "control", case + ".dat"), t / "control_file.dat")
    return tmp_path


def test_reference_test_cases_run(fz, tree):
    import torch
    from firtez_dz_b200 import control, v3io
    t = tree / "tests"
    lines = fz.lines_parse(open(tree / "default" / "lines_database.dat").read())
    reg = fz.regions_from_lines_section("4,5 500 -700.0 5.0", lines)
    ctx = fz.Synthesis(lines, reg, nz=256)
    # test_syn1: the profile file holds the direct synthesis of the model
    out = control.run(str(t / "test_syn1" / "control_file.dat"))
    assert [os.path.basename(p) for p in out] == ["syn_profile.bin"]
    ind, wave, st = v3io.read_profile(out[0])
    m = vo.model_from_cubes(v3io.read_model(str(tree / "default" / "test_atmos.bin")))
    syn, _, s0 = ctx.forward(m, hydrostatic=False)
    assert np.all(s0 == 0)
    np.testing.assert_array_equal(st, vo.stokes_from_syn(syn, 1, 1))
    np.testing.assert_allclose(wave, -700.0 + 5.0 * np.arange(500), rtol=0, atol=1e-3)
    # test_rf: the response functions to T and Bz at every height
    out = control.run(str(t / "test_rf" / "control_file.dat"))
    assert [os.path.basename(p) for p in out] == ["syn_profile.bin", "rfout_rf_test_atmos.bin"]
    _, logv, _, _, data = v3io.read_rf(out[1])
    assert list(logv) == [1, 0, 0, 0, 0, 1, 0, 0] and data.shape == (1, 1, 256, 500, 4, 2)
    mr = torch.from_numpy(vo.model_from_cubes(v3io.read_model(str(tree / "default" / "rf_test_atmos.bin")))).cuda()
    rf = torch.empty((1, 6, 256, 2000), dtype=torch.float32, device="cuda")
    so = torch.empty((1, 4, 500), dtype=torch.float64, device="cuda")
    mo = torch.empty_like(mr)
    ctx.forward_rf_full_device(mr.data_ptr(), 1, so.data_ptr(), rf.data_ptr(), mo.data_ptr(), hydrostatic=False)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(data, vo.rf_payload(rf.cpu().numpy(), 1, 1)[..., [0, 4]])
    # test_he and test_tau1: the output model's rows
    out = control.run(str(t / "test_he" / "control_file.dat"))
    he = vo.model_from_cubes(v3io.read_model(out[0]))
    mh, _ = ctx.hydrostatic(m, mode=True)
    np.testing.assert_array_equal(he[:, :5], mh[:, :5])
    out = control.run(str(t / "test_tau1" / "control_file.dat"))
    tau = vo.model_from_cubes(v3io.read_model(out[0]))
    mt, _ = ctx.log_tau5(m, hydrostatic=False)
    np.testing.assert_array_equal(tau[:, 11], mt[:, 11])
