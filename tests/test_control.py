"""The control-file host (firtez-dz_b200/control.py) on the reference's own
test cases' control files (tests/golden/control/, copied from the
reference's tests/ by tests/golden/make_fixtures.py) and on an example with
every section: the keys and defaults READ_INPUT_FILE applies, and the
inversion's node schedule (GET_NJEVALS / UPDATE_COEFS / MAXITER)."""
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CTRL = os.path.join(HERE, "golden", "control")


@pytest.fixture(scope="module")
def ctl(fz):
    from firtez_dz_b200 import control
    return control


def _read(ctl, case):
    return ctl.read(open(os.path.join(CTRL, case + ".dat")).read())


def test_reference_test_cases(ctl):
    c = _read(ctl, "test_syn1")
    assert (c.mode, c.hydrostatic, c.filemodel, c.fileprofile) == ("s", False, "test_atmos.bin", "syn_profile.bin")
    assert c.lines == "4,5 500 -700.0 5.0" and c.inv_stk == [True] * 4 and c.wstk == [1.0] * 4
    assert c.paths["MODPATH"] == "../../default/" and c.paths["OUTPATH"] == "./out_dir/"
    c = _read(ctl, "test_rf")
    assert c.save_rfs and c.nslb_max == {1: None, 6: None} and c.mode == "s"
    c = _read(ctl, "test_inv1")
    assert c.mode == "i" and c.hydrostatic and c.nslb_max == {1: None, 7: None}
    assert c.pen_typ == {1: 1, 7: 1} and c.pen_alp == {1: 0.01, 7: 0.1}
    assert (c.solver, c.node_expansion) == (2, 2) and c.paths["DATAPATH"] == "../test_syn1/out_dir/"
    # every height free for T and v_z, regularised, not progressive: only the
    # last of FLOOR(LOG(256)/LOG(2)) = 8 cycles runs, with NZ nodes each
    assert c.schedule(256) == [{1: 256, 7: 256}]
    assert _read(ctl, "test_he").mode == "h" and _read(ctl, "test_he").hydrostatic
    assert _read(ctl, "test_tau1").mode == "t"


def test_full_example_and_schedule(ctl):
    text = """
# the inversion of the benchmarked configuration
LINES:
1 112 -1193.25 21.5   # Fe I 6301.5
2 112 -1193.25 21.5
FILEPROFILE:
obs.bin
FILEMODEL:
guess.bin
MODE:
inversion
HYDROSTATIC:
yes
STOKES SETUP:
STKI 1.0
STKQ 3.0
STKU 3.0
STKV 1.6
INVERSION SETUP:
TEM 5
BX 2
BY 2
BZ 2
VLOS 2
LINE SPREAD FUNCTION:
32.35 0.
lsf2.bin
MISC SETUP:
TEMP
BVEC
PROGRESSIVE
NOISE 1e-3
SVDTOL 1e-5
END:
ignored after END
"""
    c = ctl.read(text)
    assert c.lines.splitlines() == ["1 112 -1193.25 21.5", "2 112 -1193.25 21.5"]
    assert c.mode == "i" and c.assist == {"temp", "bvec"} and c.progressive
    assert c.isigma == 1e-3 and c.svdtol == 1e-5 and c.lsf == [(32.35, 0.0), "lsf2.bin"]
    w = [1.0, 3.0, 3.0, 1.6]
    n = (sum(x * x for x in w) / 4) ** 0.5
    assert c.wstk == pytest.approx([x / n for x in w])
    # MAXITER = FLOOR(LOG(5)/LOG(2)) = 2: T on 2 nodes and the rest on 1,
    # then everything at its maximum
    assert c.schedule(128) == [{1: 2, 4: 1, 5: 1, 6: 1, 7: 1}, {1: 5, 4: 2, 5: 2, 6: 2, 7: 2}]
    # one node each: one cycle; POW 3 and 30 nodes: three cycles
    assert ctl.read("INVERSION SETUP:\nTEM 1\nBZ 1\n").schedule(64) == [{1: 1, 6: 1}]
    c3 = ctl.read("INVERSION SETUP:\nTEM 30\nVLOS 4\nPOW 3\n")
    assert c3.schedule(64) == [{1: 3, 7: 1}, {1: 9, 7: 3}, {1: 30, 7: 4}]
    # the largest count below CYCPOW: MAXITER = 0, no cycle (as the reference)
    assert ctl.read("INVERSION SETUP:\nTEM 2\nBZ 1\nPOW 3\n").schedule(64) == []
