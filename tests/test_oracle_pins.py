"""Pins of the CPU oracle against the reference's own artefacts (no GPU).

* partition functions: the table evaluator against a literal Fortran-semantics
  evaluation of src/atom_database.f90:121-1035 (tests/golden/partition_function.npz);
* chemical equilibrium GET_RHO (src/chemical_equilibrium.f90:165-278): the
  reference fixture default/test_atmos.bin carries rho, Pe and mu computed
  by the reference from its T and Pg with the abundance set that
  src/atom_database.f90:89-97 keeps commented out;
* continuum opacity at 5000 A + the log tau5 trapezoid (src/forward.f90:926,
  :1000-1006): the fixture's log tau5 was written by the reference with
  KC5 per gram (divided by MW, the `/MW(K)` left commented at :927).
"""
import os

import numpy as np
import pytest

import fixtures

MAMU = 1.66053892e-24
KBOL = 1.38056503e-16


def test_partition_function_table_matches_literal_reference(orc):
    g = np.load(os.path.join(fixtures.GOLDEN, "partition_function.npz"))
    T, U = g["T"], g["U"]
    worst_u = worst_d = 0.0
    for z in range(1, 93):
        for i in range(0, len(T), 3):
            o = orc.partition(z, T[i])
            ref = U[z - 1, i]
            worst_u = max(worst_u, np.max(np.abs(o[:3] - ref[:3]) / np.maximum(np.abs(ref[:3]), 1e-300)))
            den = np.where(np.abs(ref[3:]) > 0, np.abs(ref[3:]), 1.0)
            worst_d = max(worst_d, np.max(np.abs(o[3:] - ref[3:]) / den))
    assert worst_u == 0.0, worst_u          # bit-exact values
    assert worst_d < 1e-9, worst_d           # derivatives: evaluation order only


@pytest.fixture()
def fixture_abund(orc):
    orc.set_abundances(fixtures.fixture_abundances())
    yield
    orc.set_abundances(None)


def test_chemistry_reproduces_reference_fixture(orc, fixture_abund):
    m = fixtures.fixture_model()[0]
    T, Pg, rho, Pe, mu = m[0], m[1], m[2], m[3], m[4]
    ne = 0.0
    got = []
    for k in range(len(T)):
        r = orc.get_rho(float(T[k]), float(Pg[k]), ne)
        ne = r["nelec"]
        assert r["status"] == 0
        got.append((r["dens"], r["molecw"], ne * KBOL * float(T[k])))
    got = np.array(got)
    # rho, mu, Pe = ne k T within the fixed-point tolerance of GET_RHO (1e-4
    # per iteration; the fixture used another warm-start chain)
    assert np.max(np.abs(got[:, 0] / rho - 1)) < 5e-7
    assert np.max(np.abs(got[:, 1] / mu - 1)) < 3e-6
    assert np.max(np.abs(got[:, 2] / Pe - 1)) < 5e-7


def test_tau5_reproduces_reference_fixture(orc, fixture_abund):
    m = fixtures.fixture_model()[0]
    T, Pg, rho, mu, z, ltau = m[0], m[1], m[2], m[4], m[12].astype(np.float64), m[11]
    L = orc.lib()
    ne = 0.0
    kc5 = np.zeros(len(T))
    for k in range(len(T)):
        r = orc.get_rho(float(T[k]), float(Pg[k]), ne)
        ne = r["nelec"]
        kc5[k] = L.orc_opac_continuum(float(T[k]), 5000.0, ne, r["nhyd"]) / r["nhyd"] * (1.0 / MAMU)
    kcg = kc5 / mu.astype(np.float64)
    tau = np.zeros(len(T), np.float32)
    tau[-1] = np.float32(1e-9)
    for k in range(len(T) - 2, -1, -1):
        a = (np.float32(kcg[k]) * rho[k] + np.float32(kcg[k + 1]) * rho[k + 1]) / np.float32(2.0)
        tau[k] = np.float32(np.float64(tau[k + 1]) + np.float64(a) * ((z[k + 1] - z[k]) * 1000.0 * 100.0))
    assert np.max(np.abs(np.log10(tau) - ltau)) < 1e-6


def test_voigt_limits(orc):
    x = np.linspace(0.0, 40.0, 4001)
    v = np.concatenate([-x[::-1], x[1:]])
    h, f = orc.voigt(0.05, v)
    assert np.allclose(h, h[::-1], rtol=0, atol=0)          # H even in v
    assert np.allclose(f, -f[::-1], rtol=0, atol=0)         # F odd in v
    assert abs(np.trapezoid(h, v) / np.sqrt(np.pi) - 1) < 2e-2
    h0, _ = orc.voigt(0.0, np.array([0.0, 0.5, 1.0, 2.0]))
    assert np.allclose(h0, np.exp(-np.array([0.0, 0.5, 1.0, 2.0]) ** 2))


def test_zeeman_patterns(orc):
    lines = orc.parse_lines(fixtures.fixture_lines_text())
    ln = lines[lines["num"] == 4][0]            # Fe I 6301.5 5P2-5D2
    sh, st, ty = orc.zeeman(ln)
    assert len(sh) == 13
    for t in (-1, 0, 1):
        assert abs(st[ty == t].sum() - 1.0) < 1e-15
    ln = lines[lines["num"] == 5][0]            # Fe I 6302.5 5P1-5D0, g_eff = 2.5
    sh, st, ty = orc.zeeman(ln)
    assert len(sh) == 3
    geff = abs(sh[ty == 1][0]) / (4.66685e-10 * ln["l0"] ** 2)
    assert abs(geff - 2.5) < 1e-6


def test_generated_tables_match_a_second_parse_of_the_reference():
    """fz_tables.h (written by oracle/gen_tables.py, compiled into both the
    library and the oracle) against tests/golden/table_pins.npz, a second
    parse of the same Fortran DATA by tests/golden/make_table_pins.py that
    shares no code with the generator: the six ABO cross-section / velocity
    exponent grids (src/damping.f90:24-840) and the HSRA T, Pg, rho, z
    (src/normalization.f90:135-393), bit for bit."""
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    hdr = open(os.path.join(root, "firtez-dz_b200", "csrc", "fz_tables.h")).read()
    pins = np.load(os.path.join(root, "tests", "golden", "table_pins.npz"))

    def c_array(name):
        m = re.search(r"\b%s(\[[^=]*)=\s*\{(.*?)\};" % name, hdr, flags=re.S)
        dims = [d for d in re.findall(r"\[(\w+)\]", m.group(1))]
        nums = [float(x) for x in re.findall(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?", m.group(2))]
        return dims, np.array(nums)

    for key in pins.files:
        dims, vals = c_array("fz_tab_" + key)
        ref = pins[key]
        assert vals.size == ref.size, key
        if key.startswith("hsra"):
            assert np.array_equal(vals.astype(np.float32), ref), key
        else:
            assert [int(d) for d in dims] == list(ref.shape), key
            assert np.array_equal(vals.reshape(ref.shape), ref), key
