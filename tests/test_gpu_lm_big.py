"""The batched LM for node layouts above 16 nodes against the FP64 oracle.

The reference's default schedule frees every height of a parameter in its
last cycle; its only inversion test (tests/test_inv1) runs T and v_z at all
256 heights (NP = 512) with LINEAR_SOLVER 2, PERTURBATION_TYPE 2 and type-1
vertical regularisation.  Layouts above 16 nodes take the node Jacobian from
the response functions at every height (contracted by the hat table), the
normal equations from the tcgen05 kernel (split-bf16 x3 in tensor memory)
and the CTA-wide FP64 solvers.

* GET_PERTURBATION at NP = 40, 130 and 300 (one, two and three 128-row
  tiles): the SVD path against LAPACK DGESVD within 1e-3 of |delta| (as the
  16-node kernels), the conjugate-gradient path within the reference's own
  stopping test and 5 % of the oracle's CG delta.
* The node Jacobian of 72- and 96-node layouts against the oracle's,
  within 2e-4 of the largest entry of each parameter's node columns.
* The inversion at test_inv1's shape (NZ 256, Fe I 6301.5 blended with
  6302.5 x 500 wavelengths, T and v_z at every height, CG, STiC-like
  expansion, type-1 regularisation) run for 1, 2 and 3 iterations against
  the oracle's inversion stopped at the same iteration: the accept
  decision, lambda and STEPS exactly.  The CG stops once the mean squared
  relative residual is below 1e-3, so two FP64 runs on Hessians a few 1e-6
  apart may stop one iteration apart.  The oracle itself, its synthesis
  perturbed by 5e-7 and its Jacobian by 2e-6 (FP32 rounding), moves its
  chi2 by up to 0.2 % after the second iteration and 1.2 % after the
  third, and its node values by up to 0.2 % and 2.3 % of PARAM_NORM
  (tests/test_cg_sensitivity_cpu.py): chi2 is held within 1e-3 after the
  first iteration and 2e-2 after the later ones, the node values within
  1 % of PARAM_NORM after the first two and 3 % after the third.  With
  the SVD solver on a 64-node layout: chi2 within 1e-3 and node values
  within 1e-4 of PARAM_NORM at every iteration.
* test_inv1 itself through the control-file host.
"""
import os
import shutil
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import lm_oracle as lmo  # noqa: E402
import lmcase  # noqa: E402
import v3_oracle as vo  # noqa: E402

pytestmark = pytest.mark.gpu

NORMS = {1: 6000.0, 2: 1.0e5, 4: 1.0e3, 5: 1.0e3, 6: 1.0e3, 7: 1.0e6}


def _jac(rng, npar, nf):
    u, _ = np.linalg.qr(rng.standard_normal((nf, npar)))
    v, _ = np.linalg.qr(rng.standard_normal((npar, npar)))
    k = max(1, npar // 10)
    s = np.concatenate([np.logspace(0, -1.5, npar - k), np.full(k, 3e-3)]) * 50.0
    return ((u * s) @ v.T).T


@pytest.mark.parametrize("npar", [40, 130, 300])
def test_lm_perturbation_large_layouts(fz, orc, npar):
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    ctx = fz.Synthesis(lines, reg, nz=32)
    rng = np.random.default_rng(npar)
    npix, nf = 3, 896
    jac = np.stack([_jac(rng, npar, nf) for _ in range(npix)])
    diff = rng.standard_normal((npix, nf))
    lam = np.array([0.01, 0.3, 10.0])
    d = ctx.lm_perturbation(jac, diff, lam)
    for i in range(npix):
        ref = lmo.get_perturbation(jac[i].T, diff[i], lam[i])
        assert np.linalg.norm(d[i] - ref) <= 1e-3 * np.linalg.norm(ref), (npar, i)
    dc = ctx.lm_perturbation(jac, diff, lam, dtype=2)
    for i in range(npix):
        jn = jac[i].T
        hss = jn.T @ jn
        a = hss + np.diag(np.diag(hss)) * lam[i]
        b = jn.T @ diff[i]
        cond = np.sum(((a @ dc[i] - b) / (np.abs(b) + 1e-5)) ** 2) / npar
        assert cond < 2e-3, (npar, i, cond)
        ref = lmo.get_perturbation(jn, diff[i], lam[i], dtype=2)
        assert np.linalg.norm(dc[i] - ref) <= 5e-2 * np.linalg.norm(ref), (npar, i)


@pytest.mark.parametrize("nodes", [{1: 48, 7: 48}, {1: 24, 4: 8, 5: 8, 6: 8, 7: 24}])
def test_node_jacobian_of_large_layouts(fz, orc, nodes):
    nz = 48
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    g, _ = orc.gain(lines, reg)
    m = fz.atmos.make_columns(3, nz, seed=17)
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    np_ = ctx.rf_nodes(nodes)
    assert np_ == sum(nodes.values())
    syn, jac, _, st = ctx.forward_rf(m, hydrostatic=True)
    osyn, ojac, _, ost = orc.forward_rf(lines, reg, g, m, nodes, hydrostatic=True)
    assert np.all(st == 0) and np.all(ost == 0)
    assert np.max(np.abs(syn[:, 0] - osyn[:, 0]) / np.abs(osyn[:, 0])) < 1e-5
    # A node column of a layout with a node at every height is the RF of one
    # height, which is tiny deep in the column; the error is measured against
    # the largest entry of the parameter's node columns.
    err = np.abs(jac.astype(np.float64) - ojac).max(axis=2)
    j0 = 0
    for p, nj in sorted(nodes.items()):
        scale = np.abs(ojac[:, j0:j0 + nj]).max(axis=(1, 2))
        rel = err[:, j0:j0 + nj].max(axis=1) / np.where(scale > 0, scale, 1.0)
        assert rel.max() <= 2e-4, (p, rel.max())
        j0 += nj


def _inv1_case(fz, orc):
    gold = os.path.join(HERE, "golden")
    lines = fz.lines_parse(open(os.path.join(gold, "lines_database.dat")).read())
    reg = fz.regions_from_lines_section("4,5 500 -700.0 5.0", lines)
    g, _ = orc.gain(lines, reg)
    from firtez_dz_b200 import v3io
    m = vo.model_from_cubes(v3io.read_model(os.path.join(gold, "test_atmos.bin")))
    obs, _, _ = orc.forward(lines, reg, g, m, hydrostatic=False)
    init = m.copy()
    init[:, 0] += (150.0 * np.cos(np.linspace(0.0, 3.0, m.shape[2]))).astype(np.float32)
    init[:, 10] += 1.5e4
    return lines, reg, g, obs.reshape(1, -1), init


def _nodevals(model, nodes):
    out = []
    for p, nj in sorted(nodes.items()):
        out.append(lmo.contract(model[lmo.ATMPOS[p]], lmo.int_coefs(model.shape[1], nj)) / NORMS[p])
    return np.concatenate(out)


@pytest.mark.parametrize("solver,nz_nodes,tol", [(2, 256, 1e-2), (1, 32, 1e-4)])
def test_large_layout_iterations_match_oracle(fz, orc, solver, nz_nodes, tol):
    lines, reg, g, obs, init = _inv1_case(fz, orc)
    nz = init.shape[2]
    nodes = {1: nz_nodes, 7: nz_nodes}
    pen_typ = [1, 0, 0, 0, 0, 0, 1, 0]
    pen_alp = [0.01, 0, 0, 0, 0, 0, 0.1, 0]
    w = lmo.weights(obs.shape[1] // 4, isigma=4e-3)
    rec = []
    lmo.invert(lmcase.oracle_forward_rf(orc, lines, reg, g, True, nodes), obs, init, nodes, w, maxsteps=5, maxit=3,
               dchi2=0.0, reg=(pen_typ, pen_alp), solver=solver, node_expansion=2, record=rec)
    ctx = fz.Synthesis(lines, reg, nz=nz, gain=g)
    assert ctx.rf_nodes(nodes) == 2 * nz_nodes
    for k in (1, 2, 3):
        state = np.zeros((1, 5))
        opts = fz.LMOpts(maxsteps=5, maxit=k, dchi2=0.0, isigma=4e-3, slots=1, solver=solver, node_expansion=2,
                         reg={1: (1, 0.01), 7: (1, 0.1)}, state_out=state.ctypes.data)
        mo, chi, it, st = ctx.invert(obs.reshape(1, 4, -1), init, hydrostatic=True, opts=opts)
        steps, chicur, chibest, precyc, lam, best, acc = rec[k - 1][0]
        assert st[0] == 0 and it[0] == k
        ctol = 1e-3 if solver == 1 or k == 1 else 2e-2
        assert abs(state[0, 2] - chibest) <= ctol * chibest, (k, state[0], chibest)
        assert abs(state[0, 1] - chicur) <= ctol * chicur, (k, state[0], chicur)
        assert (state[0, 1] == state[0, 2]) == acc, k
        assert (state[0, 0], state[0, 3], state[0, 4]) == (steps, precyc, lam), (k, state[0])
        dn = np.abs(_nodevals(mo[0], nodes) - _nodevals(best, nodes))
        ntol = 3e-2 if solver == 2 and k == 3 else tol
        assert dn.max() <= ntol, (k, float(dn.max()))


def test_reference_inversion_test_case_runs(fz, tmp_path):
    """tests/test_inv1 through the control-file host: the inverted model and
    its synthesis are written, finite, and the profile file is the
    synthesis of the model file (END_CYCLE's forward pass)."""
    from firtez_dz_b200 import control, v3io
    gold = os.path.join(HERE, "golden")
    d = tmp_path / "default"
    d.mkdir()
    for f in ("test_atmos.bin", "lines_database.dat"):
        shutil.copyfile(os.path.join(gold, f), d / f)
    for case in ("test_syn1", "test_inv1"):
        t = tmp_path / "tests" / case
        (t / "out_dir").mkdir(parents=True)
        shutil.copyfile(os.path.join(gold, "control", case + ".dat"), t / "control_file.dat")
    control.run(str(tmp_path / "tests" / "test_syn1" / "control_file.dat"))
    out = control.run(str(tmp_path / "tests" / "test_inv1" / "control_file.dat"))
    assert [os.path.basename(p) for p in out] == ["out_test_atmos.bin", "out_syn_profile.bin"]
    mod = vo.model_from_cubes(v3io.read_model(out[0]))
    _, _, st = v3io.read_profile(out[1])
    assert np.all(np.isfinite(mod)) and np.all(np.isfinite(st))
    lines = fz.lines_parse(open(os.path.join(gold, "lines_database.dat")).read())
    reg = fz.regions_from_lines_section("4,5 500 -700.0 5.0", lines)
    ctx = fz.Synthesis(lines, reg, nz=256)
    syn, _, s0 = ctx.forward(mod, hydrostatic=True)
    assert np.all(s0 == 0)
    np.testing.assert_array_equal(st, vo.stokes_from_syn(syn, 1, 1))
