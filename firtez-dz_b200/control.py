"""FIRTEZ-dz's control file and a host that runs its modes through the
library -- the role of the Fortran main program (READ_MINPUT_FILE /
READ_INPUT_FILE, src/input_file.f90:43-707; INVERT3D's schedule,
src/invert3d.f90:57-178, src/get_dmodel.f90:377-442, :648-721,
src/pre_post_duties.f90:625-650) for the reference's test cases.

read(text) -> Control: the keyword sections (`KEY:` lines, values on the
following lines; blank lines, `#` comments and everything after `END:`
ignored), with the reference's defaults.  Control.schedule(nz) -> the node
counts of every inversion cycle.  run(path) executes MODE synthesis (with
WRITE RESPONSE FUNCTION), inversion, tau and hydrostatic on GPU 0 and
writes the reference's v3 files.
"""
import math
import os

import numpy as np

# INVERSION SETUP / VERTICAL REGULARIZATION keys -> reference parameter (1-based)
PARAMS = {"TEM": 1, "PGAS": 2, "RHO": 3, "BX": 4, "BY": 5, "BZ": 6, "VLOS": 7, "P0": 8}
STOKES = ("STKI", "STKQ", "STKU", "STKV")


def _number(tok):
    """GET_NUMBER: an integer or a real."""
    try:
        return int(tok)
    except ValueError:
        return float(tok)


class Control:
    """The parsed control file (fields named after the reference's variables)."""

    def __init__(self):
        self.lines = ""                 # the LINES: rows
        self.fileprofile = None
        self.filemodel = None
        self.mode = None                # 's', 'i', 't' or 'h' (first letter of MODE:)
        self.hydrostatic = False
        self.inv_stk = [False] * 4
        self.wstk = [1.0] * 4           # normalised as NSET_STK_INVERSION does
        self.nslb_max = {}              # inverted parameter -> maximum node count (None: NZ)
        self.cycpow, self.maxsteps = 2, 5
        self.pen_typ, self.pen_alp = {}, {}
        self.save_rfs = False
        self.lsf = []                   # per region: (sigma, w0) or a file name
        self.paths = {"DATAPATH": "./", "MODPATH": "./", "OUTPATH": "./", "SLDPATH": "./"}
        self.assist = set()
        self.progressive = False
        self.isigma, self.svdtol = 4.0e-3, 1.0e-4
        self.solver, self.node_expansion = 1, 1

    @property
    def vregularization(self):
        return bool(self.pen_typ) or bool(self.pen_alp)

    def schedule(self, nz):
        """Node counts {reference parameter: NJ} of every cycle INVERT3D runs:
        MAXITER = 1 when every parameter has one node, else
        FLOOR(LOG(max NSLB)/LOG(CYCPOW)); in cycle I (TOFFSET = 1) T has
        CYCPOW^I nodes, the others 1 in the first cycle and CYCPOW^(I-1) after,
        all NZ in the last, each at most its NSLB_MAX and NZ (GET_NJEVALS,
        UPDATE_COEFS); with vertical regularisation and no PROGRESSIVE only
        the last cycle runs."""
        nmax = {p: (nz if v is None else int(v)) for p, v in self.nslb_max.items()}
        if not nmax:
            return []
        if sum(nmax.values()) == len(nmax):
            maxiter = 1
        else:
            # 0 (no cycle at all) when the largest node count is below CYCPOW
            maxiter = int(math.floor(math.log(float(max(nmax.values()))) / math.log(float(self.cycpow))))
        first = maxiter if (self.vregularization and not self.progressive) else 1
        out = []
        for i in range(first, maxiter + 1):
            nodes = {}
            for p, vmax in sorted(nmax.items()):
                if p == 1:
                    nj = nz if i == maxiter else min(nz, int(self.cycpow ** i))
                else:
                    nj = 1 if i == 1 else (nz if i == maxiter else min(nz, int(self.cycpow ** (i - 1))))
                nodes[p] = min(nj, vmax)
            out.append(nodes)
        return out


def read(text):
    """Parse a control file's text (READ_MINPUT_FILE's line filter, then the
    sections READ_INPUT_FILE knows)."""
    rows = []
    for raw in text.splitlines():
        ln = raw.strip()
        if not ln or ln.startswith("#"):
            continue
        if "#" in ln:
            ln = ln[:ln.index("#")].strip()
        if ln == "END:":
            break
        rows.append(ln)
    c = Control()
    i = 0

    def section(k):
        vals = []
        while k + 1 < len(rows) and ":" not in rows[k + 1]:
            k += 1
            vals.append(rows[k])
        return vals, k

    while i < len(rows):
        key = rows[i]
        vals, j = section(i)
        if key == "LINES:":
            c.lines = "\n".join(vals)
        elif key in ("FILEPROFILE:", "FILEMODEL:", "MODE:", "HYDROSTATIC:", "WRITE RESPONSE FUNCTION:") and vals:
            v = vals[0]
            if key == "FILEPROFILE:":
                c.fileprofile = v
            elif key == "FILEMODEL:":
                c.filemodel = v
            elif key == "MODE:":
                c.mode = v[0].lower()
            elif key == "HYDROSTATIC:":
                c.hydrostatic = v[0] in "yY"
            else:
                c.save_rfs = v[0] in "yY"
        elif key == "STOKES SETUP:":
            for v in vals:
                t = v.split()
                if t[0] in STOKES:
                    s = STOKES.index(t[0])
                    c.inv_stk[s] = True
                    c.wstk[s] = float(t[1]) if len(t) > 1 else 1.0
        elif key == "INVERSION SETUP:":
            for v in vals:
                t = v.split()
                if t[0] in PARAMS:
                    c.nslb_max[PARAMS[t[0]]] = int(_number(t[1])) if len(t) > 1 else None
                elif t[0] == "POW" and len(t) > 1:
                    c.cycpow = int(_number(t[1]))
                elif t[0] == "MAXITER" and len(t) > 1:
                    c.maxsteps = int(_number(t[1]))
        elif key == "VERTICAL REGULARIZATION TYPE:":
            for v in vals:
                t = v.split()
                if t[0] in PARAMS:
                    c.pen_typ[PARAMS[t[0]]] = int(_number(t[1])) if len(t) > 1 else 0
        elif key == "VERTICAL REGULARIZATION NORM:":
            for v in vals:
                t = v.split()
                if t[0] in PARAMS:
                    c.pen_alp[PARAMS[t[0]]] = float(t[1]) if len(t) > 1 else 0.0
        elif key == "LINE SPREAD FUNCTION:":
            for v in vals:
                t = v.split()
                try:
                    c.lsf.append((float(t[0]), float(t[1])))
                except (ValueError, IndexError):
                    c.lsf.append(t[0])
        elif key == "MISC SETUP:":
            for v in vals:
                t = v.split()
                if t[0] in c.paths and len(t) > 1:
                    c.paths[t[0]] = t[1]
                elif t[0] in ("TEMP", "PGAS", "BVEC", "VLOS"):
                    c.assist.add(t[0].lower())
                elif t[0] == "PROGRESSIVE":
                    c.progressive = True
                elif t[0] == "NOISE" and len(t) > 1:
                    c.isigma = float(t[1])
                elif t[0] == "SVDTOL" and len(t) > 1:
                    c.svdtol = float(t[1])
                elif t[0] == "LINEAR_SOLVER" and len(t) > 1:
                    c.solver = int(_number(t[1]))
                elif t[0] == "PERTURBATION_TYPE" and len(t) > 1:
                    c.node_expansion = int(_number(t[1]))
        i = j + 1
    # NSET_STK_INVERSION's normalisation of the Stokes weights
    nst = sum(c.inv_stk)
    if nst:
        w = [c.wstk[s] if c.inv_stk[s] else 0.0 for s in range(4)]
        minw = math.sqrt(sum(x * x for x in w)) / math.sqrt(nst)
        c.wstk = [x / minw for x in w]
    return c


def _wave_index(ctx):
    """WAVE_INIT's WAVE [mA] and INDEX (the region's main line, A)."""
    wave, ind = [], []
    for r in ctx.regions:
        l0 = float(ctx.lines["l0"][int(r["line"][0])])
        for j in range(int(r["numwave"])):
            wave.append(float(r["wave_ini"]) + float(r["dlambda"]) * j)
            ind.append(l0)
    return np.array(ind), np.array(wave)


def run(path, device=0):
    """Run the control file at `path` (paths in it relative to its directory,
    as the reference runs from the test case's directory).  Returns the list
    of files written."""
    import torch

    from . import FzError, LMOpts, Synthesis, lines_parse, regions_from_lines_section, v3io
    base = os.path.dirname(os.path.abspath(path))
    c = read(open(path).read())
    rel = lambda key, name: os.path.join(base, c.paths[key], name)  # noqa: E731
    if c.filemodel is None or c.mode is None:
        raise FzError("the control file needs FILEMODEL: and MODE:")
    cubes = v3io.read_model(rel("MODPATH", c.filemodel))
    _, nx, ny, nz = cubes.shape
    npix = nx * ny
    dev = torch.device("cuda", device)
    d_model = v3io.model_from_cubes_device(torch.from_numpy(cubes).to(dev))
    xs = cubes[10, :, 0, 0].astype(np.float64)
    ys = cubes[11, 0, :, 0].astype(np.float64)
    written = []
    out_model = rel("OUTPATH", "out_" + c.filemodel)

    def write_model(d_m):
        v3io.write_model(out_model, v3io.cubes_from_model_device(d_m, nx, ny, xs, ys).cpu().numpy())
        written.append(out_model)

    if c.mode in "th":
        ldb = open(rel("SLDPATH", "lines_database.dat")).read()
        lines = lines_parse(ldb)
        reg = regions_from_lines_section(c.lines or "%d 1 0.0 1.0" % int(lines["num"][0]), lines)
        ctx = Synthesis(lines, reg, nz=nz, device=device)
        m = d_model.cpu().numpy()
        if c.mode == "t":
            mo, _ = ctx.log_tau5(m, hydrostatic=c.hydrostatic)
        elif c.hydrostatic:   # MODE h: FORWARD1D stops after the HE integration
            mo, _ = ctx.hydrostatic(m, mode=True)
        else:
            mo = m
        write_model(torch.from_numpy(mo).to(dev))
        return written
    lines = lines_parse(open(rel("SLDPATH", "lines_database.dat")).read())
    reg = regions_from_lines_section(c.lines, lines)
    ctx = Synthesis(lines, reg, nz=nz, device=device)
    for r, l in enumerate(c.lsf):
        if isinstance(l, tuple):
            if l[0] != -1 and l[1] != -1:
                ctx.lsf_gaussian(r, l[0], l[1])
        else:
            ctx.lsf_kernel(r, v3io.read_lsf(rel("DATAPATH", l), int(reg["numwave"][r])))
    ind, wave = _wave_index(ctx)
    numw = ctx.numw
    d_syn = torch.empty((npix, 4, numw), dtype=torch.float64, device=dev)
    if c.mode == "s":
        mo = torch.empty_like(d_model)
        ctx.forward_device(d_model.data_ptr(), npix, d_syn.data_ptr(), mo.data_ptr(), hydrostatic=c.hydrostatic)
        torch.cuda.synchronize()
        prof = rel("OUTPATH", c.fileprofile)
        v3io.write_profile(prof, ind, wave, v3io.stokes_from_syn_device(d_syn, nx, ny).cpu().numpy())
        written.append(prof)
        if c.save_rfs:
            # WRITE_RESPONSE_FUNCTIONS: the inverted parameters' responses at
            # every height (the library's: T, Pg, Bx, By, Bz, vz)
            logv = [0] * 8
            for p in c.nslb_max:
                if p in (3, 8):
                    raise FzError("response functions to rho or P0 are not provided")
                logv[p - 1] = 1
            keep = [q for q, p in enumerate((1, 2, 4, 5, 6, 7)) if logv[p - 1]]
            rf = torch.empty((npix, 6, nz, 4 * numw), dtype=torch.float32, device=dev)
            ctx.forward_rf_full_device(d_model.data_ptr(), npix, d_syn.data_ptr(), rf.data_ptr(), mo.data_ptr(),
                                       hydrostatic=c.hydrostatic)
            pay = v3io.rf_file_layout_device(rf, nx, ny)[..., keep].cpu().numpy()
            zz = cubes[12, 0, 0, :].astype(np.float64)
            rfile = rel("OUTPATH", "rfout_" + c.filemodel)
            v3io.write_rf(rfile, zz, logv, ind, wave, pay)
            written.append(rfile)
        return written
    if c.mode == "i":
        if not all(c.inv_stk):
            raise FzError("the library inverts all four Stokes parameters")
        _, _, st = v3io.read_profile(rel("DATAPATH", c.fileprofile))
        d_obs = v3io.obs_from_stokes_device(torch.from_numpy(st).to(dev))
        cycles = c.schedule(nz)
        reg_ = {p: (c.pen_typ.get(p, 0), c.pen_alp.get(p, 0.0)) for p in c.pen_alp}
        # MAKE_DECISION's field-wide stop on the mean STEPS (src/invert3d.f90:
        # 843-846) besides the per-pixel rule; 40 iterations as a safety cap
        opts = LMOpts(maxsteps=c.maxsteps, maxit=40, isigma=c.isigma, svdtol=c.svdtol, wstk=c.wstk,
                      reg=reg_ or None, assist=tuple(c.assist) + (("progressive",) if c.progressive else ()),
                      solver=c.solver, node_expansion=c.node_expansion, global_stop=True)
        mod, _, _, _ = ctx.invert_cycles(d_obs.cpu().numpy(), d_model.cpu().numpy(), nx, ny, cycles,
                                         hydrostatic=c.hydrostatic, opts=opts)
        d_m = torch.from_numpy(mod).to(dev)
        write_model(d_m)
        mo = torch.empty_like(d_m)
        ctx.forward_device(d_m.data_ptr(), npix, d_syn.data_ptr(), mo.data_ptr(), hydrostatic=c.hydrostatic)
        torch.cuda.synchronize()
        prof = rel("OUTPATH", "out_" + c.fileprofile)
        v3io.write_profile(prof, ind, wave, v3io.stokes_from_syn_device(d_syn, nx, ny).cpu().numpy())
        written.append(prof)
        return written
    raise FzError("unknown MODE: %r" % c.mode)
