"""firtez-dz B200: GPU Stokes synthesis of FIRTEZ-dz behind a C-ABI.

Host-side mirror of the reference's interface for the hot path, over ctypes:

  * ``lines_parse(text)``            -- NREAD_LINES_DATABASE (src/lines_database.f90:380)
  * ``regions_from_lines_section``   -- the LINES: section of the control file
                                        (src/input_file.f90:290-366) + WAVE_INIT
  * ``Synthesis(...).forward(model)``-- FORWARD3D/FORWARD1D (src/forward.f90:43, :857)
                                        batched over columns on one GPU
  * ``Synthesis.rf_nodes(nodes)`` and ``forward_rf(model)`` -- FORWARD1D with
                                        response functions: the node Jacobian
                                        EQVDSYN (src/forward.f90:511-681)

Arrays use the reference layouts: ``model`` is MODEL(NZ,13,ncol) REAL*4,
i.e. a C-ordered numpy array of shape (ncol, 13, nz); ``syn`` is
RSYN1D(NFREQ,ncol) REAL*8, i.e. shape (ncol, 4, numw).

The library is ``libfzb200.so`` next to this file (built by ``make`` in this
directory).  There is no CPU path: without the library or without a CUDA
device every compute call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfzb200.so")

MAXBLEND = 8

# Model parameter indices (src/atm_param.f90:38-75), 0-based
TEM, PG, RHO, PEL, MW, BX, BY, BZ, VX, VY, VZ, TAU5, ZZ = range(13)

FZ_OK, FZ_CHEM_NOCONV, FZ_NAN = 0, 1, 2
KERNELS = ("k_chain", "k_opac", "k_synth", "k_opac_rf", "k_synth_rf", "k_lm_fill", "k_lm_accept", "k_lm_normal",
           "k_lm_solve", "k_lm_update", "k_chemder", "k_rf_prop", "k_lsf", "k_saha",
           "k_chain_pre")

# free-parameter indices of the reference (atm_param.f90 order, 1-based) that
# carry response functions
RF_PARAMS = {1: "T", 2: "Pg", 4: "Bx", 5: "By", 6: "Bz", 7: "vz"}

LINE_DTYPE = np.dtype([
    ("num", "<i4"), ("zn", "<i4"), ("ion", "<i4"), ("flag", "<i4"), ("otr", "<i4", 2),
    ("abo_ierr", "<i4"), ("pad", "<i4"),
    ("l0", "<f8"), ("loggf", "<f8"), ("eplow", "<f8"), ("alpha", "<f8"), ("sigma", "<f8"),
    ("sl", "<f8"), ("ll", "<f8"), ("jl", "<f8"), ("su", "<f8"), ("lu", "<f8"), ("ju", "<f8"),
    ("elowlim", "<f8"), ("eupplim", "<f8"),
], align=True)

REGION_DTYPE = np.dtype([
    ("nblend", "<i4"), ("line", "<i4", MAXBLEND), ("wdif", "<f8", MAXBLEND),
    ("numwave", "<i4"), ("pad", "<i4"), ("wave_ini", "<f8"), ("dlambda", "<f8"),
], align=True)


class FzError(RuntimeError):
    pass


class LMOpts(ctypes.Structure):
    """fz_lm_opts: stop rules and weights of the batched inversion."""
    _fields_ = [("maxsteps", ctypes.c_int), ("maxit", ctypes.c_int), ("dchi2", ctypes.c_double),
                ("svdtol", ctypes.c_double), ("isigma", ctypes.c_double), ("wstk", ctypes.c_float * 4),
                ("slots", ctypes.c_int), ("assist", ctypes.c_int), ("fallback", ctypes.c_double),
                ("fallback_model", ctypes.c_void_p), ("reg_type", ctypes.c_int * 8), ("reg_alpha", ctypes.c_double * 8),
                ("fallback_steps", ctypes.c_int), ("solver", ctypes.c_int), ("node_expansion", ctypes.c_int),
                ("global_stop", ctypes.c_int), ("cycles_left", ctypes.c_int), ("fallback_free", ctypes.c_int),
                ("state_out", ctypes.c_void_p)]

    def __init__(self, maxsteps=5, maxit=40, dchi2=0.0, svdtol=1e-4, isigma=4e-3, wstk=(1, 1, 1, 1), slots=0,
                 fallback=0.0, fallback_model=0, reg=None, assist=(), fallback_steps=0, solver=1, node_expansion=1,
                 global_stop=False, cycles_left=0, state_out=0, fallback_free=False):
        """fallback_model: device pointer of one MODEL(NZ,13) float32 (e.g. a
        torch tensor's data_ptr()) that pixels ending above fallback x their
        chi2 goal restart from (a host pointer for invert()).  reg: optional
        {reference parameter: (type, alpha)} vertical regularisation
        (VERTICAL REGULARIZATION: type 0 or 1, PEN_ALP).  assist: SET_TAU's
        assists for invert_cycles (temp, pgas, bvec, vlos, progressive).
        fallback_steps: restart once STEPS reaches it while above fallback x
        the goal (0: when the search ends; negative: at the first
        evaluation); fallback_free: the restarted search ignores the goal.
        solver: 1 SVD, 2 conjugate
        gradients (LINEAR_SOLVER); node_expansion: 1 SIR-like, 2 STiC-like
        (PERTURBATION_TYPE).  global_stop: MAKE_DECISION's field-wide stop on
        the mean STEPS (threshold max(1, maxsteps - cycles_left)); state_out:
        pointer of a (npix, 5) float64 array receiving each pixel's final
        STEPS, chi2 of its last model, best chi2, PRECYC and lambda (device
        pointer for the device calls, host pointer for invert())."""
        typ, alp = [0] * 8, [0.0] * 8
        for p, (t, a) in (reg or {}).items():
            typ[int(p) - 1], alp[int(p) - 1] = int(t), float(a)
        super().__init__(maxsteps, maxit, dchi2, svdtol, isigma, (ctypes.c_float * 4)(*wstk), slots,
                         assist_bits(assist),
                         float(fallback), fallback_model or None, (ctypes.c_int * 8)(*typ),
                         (ctypes.c_double * 8)(*alp), int(fallback_steps), int(solver), int(node_expansion),
                         int(bool(global_stop)), int(cycles_left), int(bool(fallback_free)), state_out or None)


class Tune(ctypes.Structure):
    """fz_tune: launch shapes chosen by the autotuner (and their timings)."""
    _fields_ = [("chain_warps", ctypes.c_int), ("chemder_blocks_per_sm", ctypes.c_int),
                ("opac_rf_threads", ctypes.c_int), ("lm_slots", ctypes.c_int), ("chain_ms", ctypes.c_float),
                ("chemder_ms", ctypes.c_float), ("opac_rf_ms", ctypes.c_float), ("lm_pixels_per_s", ctypes.c_float),
                ("chain_lanes", ctypes.c_int), ("pad", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def build():
    """Compile libfzb200.so for sm_100a (nvcc cross-compiles without a GPU)."""
    import subprocess
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    """The loaded CUDA library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FzError("libfzb200.so not built (run make in %s)" % HERE)
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.fz_version.restype = ctypes.c_int
        L.fz_strerror.restype = ctypes.c_char_p
        L.fz_strerror.argtypes = [ctypes.c_int]
        L.fz_lines_parse.argtypes = [ctypes.c_char_p, P, ctypes.c_int]
        L.fz_create.argtypes = [ctypes.POINTER(P), P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int, P, ctypes.c_int]
        L.fz_destroy.argtypes = [P]
        L.fz_numw.argtypes = [P]
        L.fz_get_gain.argtypes = [P, P]
        L.fz_forward.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, P, P]
        L.fz_forward_device.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, P, P, P]
        L.fz_forward_device_static.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, P, P, P]
        L.fz_profile_enable.argtypes = [P, ctypes.c_int]
        L.fz_profile_read.argtypes = [P, P, P, P, ctypes.c_int]
        L.fz_measure_fp32_peak.argtypes = [ctypes.c_int, P]
        L.fz_rf_nodes.argtypes = [P, P]
        L.fz_forward_rf.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, P, P, P]
        L.fz_forward_rf_device.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, P, P, P, P]
        L.fz_forward_rf_full.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, P, P, P]
        L.fz_smooth.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P]
        L.fz_smooth_device.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P]
        L.fz_smooth_shard_device.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
        L.fz_invert_cycles_device.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int, P, ctypes.c_int, P,
                                              P, P, P, P]
        L.fz_errors.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int, P, P, P, P]
        I, S = ctypes.c_int, ctypes.c_char_p
        L.fz_v3_header.argtypes = [S, P, P, P, P]
        L.fz_v3_read_model.argtypes = [S, I, I, I, P]
        L.fz_v3_write_model.argtypes = [S, I, I, I, P]
        L.fz_v3_read_profiles.argtypes = [S, I, I, I, P, P, P]
        L.fz_v3_write_profiles.argtypes = [S, I, I, I, P, P, P]
        L.fz_v3_write_rfs.argtypes = [S, I, I, I, I, P, P, P, P, P]
        L.fz_v3_read_rfs.argtypes = [S, I, I, I, I, P, P, P, P, P]
        L.fz_model_from_v3_device.argtypes = [I, I, I, P, P, P]
        L.fz_v3_read_lsf.argtypes = [S, I, P]
        L.fz_v3_write_lsf.argtypes = [S, I, P]
        L.fz_lsf_gaussian.argtypes = [P, I, ctypes.c_double, ctypes.c_double]
        L.fz_lsf_kernel.argtypes = [P, I, P, I]
        L.fz_lsf_clear.argtypes = [P]
        L.fz_hydrostatic.argtypes = [P, I, P, I, P, P]
        L.fz_hydrostatic_device.argtypes = [P, I, P, I, P, P, P]
        L.fz_log_tau5.argtypes = [P, I, P, I, P, P]
        L.fz_log_tau5_device.argtypes = [P, I, P, I, P, P, P]
        L.fz_set_tau.argtypes = [P, I, I, P, P, I, I]
        L.fz_set_tau_device.argtypes = [P, I, I, P, P, I, I, P]
        L.fz_model_to_v3_device.argtypes = [I, I, I, P, P, P, P, P]
        L.fz_obs_from_v3_device.argtypes = [I, I, P, P, P]
        L.fz_syn_to_v3_device.argtypes = [I, I, P, P, P]
        L.fz_rf_to_v3_device.argtypes = [I, I, I, P, P, P]
        L.fz_errors_device.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int, P, P, P, P, P]
        L.fz_autotune_forward.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P]
        L.fz_autotune_lm.argtypes = [P, ctypes.c_int, P, P, P, ctypes.c_int, P, P, ctypes.c_int, P]
        L.fz_tune_get.argtypes = [P, P]
        L.fz_tune_set.argtypes = [P, P]
        L.fz_forward_rf_full_device.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, P, P, P, P]
        L.fz_invert.argtypes = [P, ctypes.c_int, P, P, P, ctypes.c_int, P, P, P, P, P, P]
        L.fz_invert_device.argtypes = [P, ctypes.c_int, P, P, P, ctypes.c_int, P, P, P, P, P, P, P]
        L.fz_lm_perturbation.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P, P, P, ctypes.c_int,
                                         ctypes.c_double, P]
        L.fz_lm_perturbation_f32.argtypes = L.fz_lm_perturbation.argtypes
        L.fz_lm_update_lambda.argtypes = [ctypes.c_int, P, P, P, P, P]
        L.fz_lm_rearange.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int]
        L.fz_lm_rearange_device.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int, P]
        L.fz_rte_solve.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P, P, P]
        L.fz_voigt.argtypes = [ctypes.c_int, P, P, P, P]
        _lib = L
    return _lib


ASSIST = {"temp": 1, "pgas": 2, "bvec": 4, "vlos": 8, "progressive": 16}


def assist_bits(names):
    """FZ_ASSIST_* bits of assist names (temp, pgas, bvec, vlos, progressive)."""
    b = 0
    for n in names or ():
        b |= ASSIST[n.lower()]
    return b


def he_mode(hydrostatic):
    """FZ_HE_* of a hydrostatic argument: False/0 Pg given, True/1 from the
    top (HYDRO_TOP), "ltau"/2 from the height of least |log tau5|."""
    if isinstance(hydrostatic, str):
        return {"none": 0, "top": 1, "ltau": 2}[hydrostatic]
    return 2 if hydrostatic == 2 else int(bool(hydrostatic))


def _check(rc):
    if rc < 0:
        raise FzError(lib().fz_strerror(rc).decode())
    return rc


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def lines_parse(text):
    """Parse lines_database.dat text into a LINE_DTYPE array."""
    out = np.zeros(512, dtype=LINE_DTYPE)
    n = _check(lib().fz_lines_parse(text.encode(), _p(out), len(out)))
    return out[:n].copy()


def regions_from_lines_section(section, lines):
    """Regions from LINES: rows like ``4,5 500 -700.0 5.0``.

    First field: database ids of the main line and its blends (comma
    separated); then NUMWAVE, WAVE_INI [mA] and DELTA_LAMBDA [mA].  BLENDSDIFF
    is 1e3*(lambda_blend - lambda_main) [mA] (src/input_file.f90:346-354)."""
    ids = {int(n): i for i, n in enumerate(lines["num"])}
    rows = [r.split() for r in section.strip().splitlines() if r.strip() and not r.strip().startswith("#")]
    reg = np.zeros(len(rows), dtype=REGION_DTYPE)
    for k, f in enumerate(rows):
        nums = [int(x) for x in f[0].split(",") if x]
        if len(nums) > MAXBLEND:
            raise ValueError("too many blends")
        reg["nblend"][k] = len(nums)
        for b, n in enumerate(nums):
            if n not in ids:
                raise ValueError("line %d is not in the database" % n)
            reg["line"][k, b] = ids[n]
            if b > 0:
                reg["wdif"][k, b] = 1.0e3 * (lines["l0"][ids[n]] - lines["l0"][ids[nums[0]]])
        reg["numwave"][k] = int(f[1])
        reg["wave_ini"][k] = float(f[2])
        reg["dlambda"][k] = float(f[3])
    return reg


class Synthesis:
    """A GPU synthesis context for one line set and height count."""

    def __init__(self, lines, regions, nz, gain=None, device=0):
        self.lines = np.ascontiguousarray(lines, dtype=LINE_DTYPE)
        self.regions = np.ascontiguousarray(regions, dtype=REGION_DTYPE)
        self.nz = int(nz)
        self.numw = int(self.regions["numwave"].sum())
        h = ctypes.c_void_p()
        g = None if gain is None else np.ascontiguousarray(gain, dtype=np.float32).reshape(self.numw, 4)
        _check(lib().fz_create(ctypes.byref(h), _p(self.lines), len(self.lines), _p(self.regions),
                               len(self.regions), self.nz, None if g is None else _p(g), int(device)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().fz_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def gain(self):
        """GAIN1D(4,NUMW) as a (numw, 4) float32 array."""
        g = np.zeros((self.numw, 4), dtype=np.float32)
        _check(lib().fz_get_gain(self._h, _p(g)))
        return g

    def forward(self, model, hydrostatic=False):
        """Synthesise host-resident columns.  model: (ncol, 13, nz) float32.

        Returns (syn (ncol, 4, numw) float64, model_out, status (ncol,))."""
        m = np.ascontiguousarray(model, dtype=np.float32)
        if m.ndim == 2:
            m = m[None]
        ncol, npar, nz = m.shape
        if npar != 13 or nz != self.nz:
            raise ValueError("model must be (ncol, 13, %d)" % self.nz)
        syn = np.zeros((ncol, 4, self.numw))
        mo = np.empty_like(m)
        st = np.zeros(ncol, dtype=np.int32)
        _check(lib().fz_forward(self._h, ncol, _p(m), he_mode(hydrostatic), _p(syn), _p(mo), _p(st)))
        return syn, mo, st

    def forward_device_static(self, model_ptr, ncol, syn_ptr, model_out_ptr, status_ptr=0, stream=0,
                              hydrostatic=False):
        """forward_device without any device allocation: the per-call scratch is
        a 64 MiB static device array (batches larger than it are rejected).
        For callers that must not allocate device memory during a call."""
        _check(lib().fz_forward_device_static(self._h, int(ncol), ctypes.c_void_p(model_ptr), he_mode(hydrostatic),
                                              ctypes.c_void_p(syn_ptr), ctypes.c_void_p(model_out_ptr),
                                              ctypes.c_void_p(status_ptr) if status_ptr else None,
                                              ctypes.c_void_p(stream) if stream else None))

    def profile(self, on=True):
        _check(lib().fz_profile_enable(self._h, int(bool(on))))

    def profile_read(self, items=False):
        """{kernel: (total ms, launches[, columns or slots processed])} since
        the last read."""
        nk = len(KERNELS)
        ms = np.zeros(nk)
        n = np.zeros(nk, dtype=np.int32)
        it = np.zeros(nk, dtype=np.int64)
        _check(lib().fz_profile_read(self._h, _p(ms), _p(n), _p(it), nk))
        if items:
            return {k: (ms[i], int(n[i]), int(it[i])) for i, k in enumerate(KERNELS)}
        return {k: (ms[i], int(n[i])) for i, k in enumerate(KERNELS)}

    def rf_nodes(self, nodes):
        """Select the free parameters of the response functions.

        nodes: {reference parameter (1 T, 2 Pg, 4 Bx, 5 By, 6 Bz, 7 vz): node
        count}; a count equal to nz gives the response at every height.
        Returns NP, the number of Jacobian columns."""
        v = np.zeros(8, dtype=np.int32)
        for p, n in nodes.items():
            if not 1 <= int(p) <= 8:
                raise ValueError("parameter index %r out of range" % p)
            v[int(p) - 1] = int(n)
        self.np = _check(lib().fz_rf_nodes(self._h, _p(v)))
        return self.np

    def forward_rf(self, model, hydrostatic=False):
        """Synthesis plus the node Jacobian of host-resident columns.

        Returns (syn (ncol, 4, numw) float64, jac (ncol, NP, 4*numw) float32 --
        EQVDSYN(NFREQ, NP) per column --, model_out, status)."""
        m = np.ascontiguousarray(model, dtype=np.float32)
        if m.ndim == 2:
            m = m[None]
        ncol, npar, nz = m.shape
        if npar != 13 or nz != self.nz:
            raise ValueError("model must be (ncol, 13, %d)" % self.nz)
        if not getattr(self, "np", 0):
            raise FzError("call rf_nodes() first")
        syn = np.zeros((ncol, 4, self.numw))
        jac = np.zeros((ncol, self.np, 4 * self.numw), dtype=np.float32)
        mo = np.empty_like(m)
        st = np.zeros(ncol, dtype=np.int32)
        _check(lib().fz_forward_rf(self._h, ncol, _p(m), he_mode(hydrostatic), _p(syn), _p(jac), _p(mo), _p(st)))
        return syn, jac, mo, st

    def forward_rf_full(self, model, hydrostatic=False):
        """Synthesis plus the response functions at every height of
        host-resident columns.

        Returns (syn (ncol, 4, numw) float64, rf (ncol, 6, nz, 4*numw) float32
        -- parameters T, Pg, Bx, By, Bz, v_z; the EQVDSYN layout with one node
        per height --, model_out, status)."""
        m = np.ascontiguousarray(model, dtype=np.float32)
        if m.ndim == 2:
            m = m[None]
        ncol, npar, nz = m.shape
        if npar != 13 or nz != self.nz:
            raise ValueError("model must be (ncol, 13, %d)" % self.nz)
        syn = np.zeros((ncol, 4, self.numw))
        rf = np.zeros((ncol, 6, self.nz, 4 * self.numw), dtype=np.float32)
        mo = np.empty_like(m)
        st = np.zeros(ncol, dtype=np.int32)
        _check(lib().fz_forward_rf_full(self._h, ncol, _p(m), he_mode(hydrostatic), _p(syn), _p(rf), _p(mo),
                                        _p(st)))
        return syn, rf, mo, st

    def forward_rf_full_device(self, model_ptr, ncol, syn_ptr, rf_ptr, model_out_ptr, status_ptr=0, stream=0,
                               hydrostatic=False):
        """Enqueue synthesis + response functions at every height on device
        pointers (rf: ncol * 6 * nz * 4 * numw float32)."""
        _check(lib().fz_forward_rf_full_device(self._h, int(ncol), ctypes.c_void_p(model_ptr),
                                               int(bool(hydrostatic)), ctypes.c_void_p(syn_ptr),
                                               ctypes.c_void_p(rf_ptr), ctypes.c_void_p(model_out_ptr),
                                               ctypes.c_void_p(status_ptr) if status_ptr else None,
                                               ctypes.c_void_p(stream) if stream else None))

    def autotune_forward(self, model_ptr, ncol, hydrostatic=True):
        """Time the launch-shape candidates of the RF path's chemistry and
        opacity kernels on ncol device columns and keep the fastest; returns
        the chosen shapes (dict)."""
        t = Tune()
        _check(lib().fz_autotune_forward(self._h, int(ncol), ctypes.c_void_p(model_ptr), int(bool(hydrostatic)),
                                         ctypes.byref(t)))
        return t.as_dict()

    def autotune_lm(self, npix, obs_ptr, init_ptr, candidates=(2048, 4096, 8192, 16384), hydrostatic=True,
                    opts=None, target_ptr=0):
        """Invert the same npix device pixels once per candidate slot count
        and keep the fastest as the default; returns the chosen shapes."""
        t = Tune()
        c = np.ascontiguousarray(candidates, dtype=np.int32)
        opts = opts or LMOpts()
        _check(lib().fz_autotune_lm(self._h, int(npix), ctypes.c_void_p(obs_ptr), ctypes.c_void_p(init_ptr),
                                    ctypes.c_void_p(target_ptr) if target_ptr else None, int(bool(hydrostatic)),
                                    ctypes.byref(opts), _p(c), int(c.size), ctypes.byref(t)))
        return t.as_dict()

    def tune(self, **shapes):
        """Current launch shapes; keyword arguments set them first."""
        t = Tune()
        _check(lib().fz_tune_get(self._h, ctypes.byref(t)))
        if shapes:
            for k, v in shapes.items():
                setattr(t, k, int(v))
            _check(lib().fz_tune_set(self._h, ctypes.byref(t)))
        d = t.as_dict()
        return {k: d[k] for k in ("chain_warps", "chain_lanes", "chemder_blocks_per_sm", "opac_rf_threads", "lm_slots")}

    def smooth(self, models, nx, ny, params=None):
        """SMOOTHING_B of host models (ny*nx, 13, nz), pixel iy + ny*ix,
        in a new array; params: iterable of reference parameters (1..8), None
        = the free parameters of rf_nodes()."""
        m = np.array(models, dtype=np.float32, order="C", copy=True)
        if m.shape != (nx * ny, 13, self.nz):
            raise ValueError("models must be (nx*ny, 13, nz)")
        f = None
        if params is not None:
            f = np.zeros(8, dtype=np.int32)
            for p in params:
                f[int(p) - 1] = 1
        _check(lib().fz_smooth(self._h, int(nx), int(ny), _p(m), None if f is None else _p(f)))
        return m

    def smooth_device(self, models_ptr, nx, ny, params=None, stream=0):
        """SMOOTHING_B in place on device models (see smooth())."""
        f = None
        if params is not None:
            f = np.zeros(8, dtype=np.int32)
            for p in params:
                f[int(p) - 1] = 1
        _check(lib().fz_smooth_device(self._h, int(nx), int(ny), ctypes.c_void_p(models_ptr),
                                      None if f is None else _p(f), ctypes.c_void_p(stream) if stream else None))

    def set_tau(self, obs, models, nx, ny, assist=("temp", "bvec", "vlos"), hydrostatic=True):
        """SET_TAU's assists on host arrays: obs (nx*ny, 4, numw), models
        (nx*ny, 13, nz) (pixel iy + ny*ix); assist: names among temp, pgas,
        bvec, vlos.  Returns the assisted models."""
        o = np.ascontiguousarray(obs, dtype=np.float64)
        m = np.array(models, dtype=np.float32, order="C", copy=True)
        if o.shape != (nx * ny, 4, self.numw) or m.shape != (nx * ny, 13, self.nz):
            raise ValueError("obs must be (nx*ny, 4, numw) and models (nx*ny, 13, nz)")
        _check(lib().fz_set_tau(self._h, int(nx), int(ny), _p(o), _p(m), assist_bits(assist), int(bool(hydrostatic))))
        return m

    def set_tau_device(self, nx, ny, obs_ptr, models_ptr, assist=("temp", "bvec", "vlos"), hydrostatic=True, stream=0):
        """SET_TAU's assists in place on device models (see set_tau())."""
        _check(lib().fz_set_tau_device(self._h, int(nx), int(ny), ctypes.c_void_p(obs_ptr),
                                       ctypes.c_void_p(models_ptr), assist_bits(assist), int(bool(hydrostatic)),
                                       ctypes.c_void_p(stream) if stream else None))

    def hydrostatic(self, model, mode=True):
        """MODE h: hydrostatic equilibrium only (mode True/"top" or "ltau").
        Returns (model_out, status)."""
        return self._model_only(model, mode, lib().fz_hydrostatic)

    def log_tau5(self, model, hydrostatic=False):
        """MODE t: log tau5 (and the chemistry rows) without the synthesis.
        Returns (model_out, status)."""
        return self._model_only(model, hydrostatic, lib().fz_log_tau5)

    def _model_only(self, model, he, fn):
        m = np.ascontiguousarray(model, dtype=np.float32)
        if m.ndim != 3 or m.shape[1:] != (13, self.nz):
            raise ValueError("model must be (ncol, 13, %d)" % self.nz)
        mo = np.empty_like(m)
        st = np.zeros(m.shape[0], dtype=np.int32)
        _check(fn(self._h, m.shape[0], _p(m), he_mode(he), _p(mo), _p(st)))
        return mo, st

    def lsf_gaussian(self, region, sigma, w0=0.0):
        """The reference's Gaussian line spread function (sigma, centre w0 in
        mA) for spectral region `region` (0-based); returns True if valid."""
        return bool(_check(lib().fz_lsf_gaussian(self._h, int(region), float(sigma), float(w0))))

    def lsf_kernel(self, region, yk):
        """A line spread function as an LSF file holds it (NUMWAVE values of
        the region, index 0 = centre); returns True if valid."""
        k = np.ascontiguousarray(yk, dtype=np.float64)
        return bool(_check(lib().fz_lsf_kernel(self._h, int(region), _p(k), k.size)))

    def lsf_clear(self):
        _check(lib().fz_lsf_clear(self._h))

    def errors(self, obs, models, hydrostatic=True, opts=None):
        """The errors mode for host models (npix, 13, nz) against obs (npix,
        4, numw) with the node layout of rf_nodes(): returns (err (npix, 13,
        nz) float32, chi2 (npix,), status (npix,)); err rows of parameters
        without nodes are zero.  opts: isigma, wstk, reg."""
        o = np.ascontiguousarray(obs, dtype=np.float64)
        m = np.ascontiguousarray(models, dtype=np.float32)
        npix = o.shape[0]
        if o.shape[1:] != (4, self.numw) or m.shape != (npix, 13, self.nz):
            raise ValueError("obs must be (npix, 4, numw) and models (npix, 13, nz)")
        err = np.zeros_like(m)
        chi = np.zeros(npix)
        st = np.zeros(npix, dtype=np.int32)
        opts = opts or LMOpts()
        _check(lib().fz_errors(self._h, npix, _p(o), _p(m), int(bool(hydrostatic)), ctypes.byref(opts), _p(err),
                               _p(chi), _p(st)))
        return err, chi, st

    def errors_device(self, npix, obs_ptr, models_ptr, err_ptr, chi2_ptr, status_ptr=0, hydrostatic=True,
                      opts=None, stream=0):
        """The errors mode on device pointers (see errors())."""
        opts = opts or LMOpts()
        _check(lib().fz_errors_device(self._h, int(npix), ctypes.c_void_p(obs_ptr), ctypes.c_void_p(models_ptr),
                                      int(bool(hydrostatic)), ctypes.byref(opts), ctypes.c_void_p(err_ptr),
                                      ctypes.c_void_p(chi2_ptr),
                                      ctypes.c_void_p(status_ptr) if status_ptr else None,
                                      ctypes.c_void_p(stream) if stream else None))

    def smooth_shard_device(self, models_ptr, nx, ny, x0, nx_field, params=None, stream=0):
        """SMOOTHING_B of a shard (columns x0 .. x0+nx-1 of an nx_field-column
        field, halo columns included) in place on device models."""
        f = None
        if params is not None:
            f = np.zeros(8, dtype=np.int32)
            for p in params:
                f[int(p) - 1] = 1
        _check(lib().fz_smooth_shard_device(self._h, int(nx), int(ny), int(x0), int(nx_field),
                                            ctypes.c_void_p(models_ptr), None if f is None else _p(f),
                                            ctypes.c_void_p(stream) if stream else None))

    def invert_cycles(self, obs, init, nx, ny, cycles, hydrostatic=True, opts=None):
        """INVERT3D's cycles on host arrays: obs (ny*nx, 4, numw), init
        (ny*nx, 13, nz) (pixel iy + ny*ix), cycles = list of node layouts
        ({reference parameter: NJ}).  Returns (final models, chi2, iterations,
        status) of the last cycle; the context keeps its node layout."""
        import torch
        npix = nx * ny
        o = np.ascontiguousarray(obs, dtype=np.float64)
        m = np.ascontiguousarray(init, dtype=np.float32)
        if o.shape != (npix, 4, self.numw) or m.shape != (npix, 13, self.nz):
            raise ValueError("obs must be (nx*ny, 4, numw) and init (nx*ny, 13, nz)")
        nodes = np.zeros((len(cycles), 8), dtype=np.int32)
        for c, lay in enumerate(cycles):
            for p, n in lay.items():
                nodes[c, int(p) - 1] = int(n)
        d_o = torch.from_numpy(o).cuda()
        d_m = torch.from_numpy(m.copy()).cuda()
        chi = torch.zeros(npix, dtype=torch.float64, device="cuda")
        it = torch.zeros(npix, dtype=torch.int32, device="cuda")
        st = torch.zeros(npix, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        opts = opts or LMOpts()
        _check(lib().fz_invert_cycles_device(self._h, int(nx), int(ny), ctypes.c_void_p(d_o.data_ptr()),
                                             ctypes.c_void_p(d_m.data_ptr()), len(cycles), _p(nodes),
                                             int(bool(hydrostatic)), ctypes.byref(opts),
                                             ctypes.c_void_p(chi.data_ptr()), ctypes.c_void_p(it.data_ptr()),
                                             ctypes.c_void_p(st.data_ptr()), None))
        self.np = int(nodes[-1].sum())
        return d_m.cpu().numpy(), chi.cpu().numpy(), it.cpu().numpy(), st.cpu().numpy()

    def invert(self, obs, init, hydrostatic=True, opts=None, want_syn=False, target=None, out=None):
        """Batched LM inversion of host-resident pixels with the node layout of
        rf_nodes().  obs: (npix, 4, numw) float64 GAIN-normalised Stokes;
        init: (npix, 13, nz) float32 initial models; target: optional
        per-pixel chi2 goal (npix,); out: optional preallocated (models,
        chi2, iterations, status) host arrays (e.g. in pinned memory).
        Returns (best models, chi2, iterations, status[, best synthesis])."""
        o = np.ascontiguousarray(obs, dtype=np.float64)
        m = np.ascontiguousarray(init, dtype=np.float32)
        npix = o.shape[0]
        if o.shape[1:] != (4, self.numw) or m.shape != (npix, 13, self.nz):
            raise ValueError("obs must be (npix, 4, numw) and init (npix, 13, nz)")
        tg = None
        if target is not None:
            tg = np.ascontiguousarray(target, dtype=np.float64)
            if tg.shape != (npix,):
                raise ValueError("target must be (npix,)")
        opts = opts or LMOpts()
        if out is not None:
            mo, chi, it, st = out
            if (mo.shape != m.shape or mo.dtype != np.float32 or chi.shape != (npix,) or chi.dtype != np.float64
                    or it.shape != (npix,) or it.dtype != np.int32 or st.shape != (npix,) or st.dtype != np.int32
                    or not all(a.flags.c_contiguous for a in (mo, chi, it, st))):
                raise ValueError("out must be contiguous (model float32, chi2 float64, iters int32, status int32)")
        else:
            mo = np.empty_like(m)
            chi = np.zeros(npix)
            it = np.zeros(npix, dtype=np.int32)
            st = np.zeros(npix, dtype=np.int32)
        syn = np.zeros_like(o) if want_syn else None
        _check(lib().fz_invert(self._h, npix, _p(o), _p(m), None if tg is None else _p(tg), int(bool(hydrostatic)),
                               ctypes.byref(opts), _p(mo),
                               _p(chi), _p(it), None if syn is None else _p(syn), _p(st)))
        return (mo, chi, it, st, syn) if want_syn else (mo, chi, it, st)

    def set_tau_shard_device(self, nx, ny, obs_ptr, models_ptr, assist, reduce, hydrostatic=True, stream=0):
        """fz_set_tau_shard_device: SET_TAU on a shard of a field split by x,
        the field sums and maxima through reduce(kind, data, n, nx) on a
        numpy view of the library's buffer (see parallel.FieldShard)."""
        L = lib()
        if not hasattr(L, "_reduce_t"):
            L._reduce_t = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                           ctypes.c_int, ctypes.c_int)
            L.fz_set_tau_shard_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_int, ctypes.c_int, L._reduce_t,
                                                  ctypes.c_void_p, ctypes.c_void_p]

        def cb(user, kind, data, n, nx_):
            try:
                view = np.ctypeslib.as_array(data, shape=(max(n * nx_, 3),))
                return int(reduce(int(kind), view, int(n), int(nx_)))
            except Exception:
                return -1

        fn = L._reduce_t(cb)
        _check(L.fz_set_tau_shard_device(self._h, int(nx), int(ny), ctypes.c_void_p(obs_ptr),
                                         ctypes.c_void_p(models_ptr), assist_bits(assist) if not isinstance(assist, int)
                                         else int(assist), int(bool(hydrostatic)), fn, None,
                                         ctypes.c_void_p(stream) if stream else None))

    def invert_warm(self, obs, warm, base=None, hydrostatic=True, opts=None, target=None, out=None):
        """fz_invert_warm: the learned initial guess and the batched LM from
        host observations (npix, 4, numw) float64, which cross to the device
        once; warm is a trained warmstart.WarmStart for this node layout,
        base one MODEL(NZ,13) (default: warmstart.default_models).  out:
        optional (models, chi2, iterations, status) host arrays.  Returns
        (models, chi2, iterations, status)."""
        from . import warmstart as ws
        ws._bind()
        o = np.ascontiguousarray(obs, dtype=np.float64)
        npix = o.shape[0]
        if o.shape[1:] != (4, self.numw):
            raise ValueError("obs must be (npix, 4, numw)")
        b = np.ascontiguousarray(ws.default_models(1, self.nz)[0] if base is None else base, dtype=np.float32)
        if getattr(warm, "_hnorm", None) is None:
            warm._hnorm = warm.norm()
        tg = None if target is None else np.ascontiguousarray(target, dtype=np.float64)
        if out is None:
            out = (np.empty((npix, 13, self.nz), dtype=np.float32), np.zeros(npix), np.zeros(npix, dtype=np.int32),
                   np.zeros(npix, dtype=np.int32))
        mo, chi, it, st = out
        opts = opts or LMOpts()
        _check(lib().fz_invert_warm(self._h, warm.mlp._h, _p(warm._hnorm), _p(b), npix, _p(o),
                                    None if tg is None else _p(tg), int(bool(hydrostatic)), ctypes.byref(opts),
                                    _p(mo), _p(chi), _p(it), None, _p(st)))
        return mo, chi, it, st

    def invert_device(self, npix, obs_ptr, init_ptr, model_out_ptr, chi2_ptr, iters_ptr, status_ptr=0, syn_ptr=0,
                      hydrostatic=True, opts=None, stream=0, target_ptr=0):
        """Batched LM inversion on device pointers (target_ptr: optional
        per-pixel chi2 goal, float64)."""
        opts = opts or LMOpts()
        _check(lib().fz_invert_device(self._h, int(npix), ctypes.c_void_p(obs_ptr), ctypes.c_void_p(init_ptr),
                                      ctypes.c_void_p(target_ptr) if target_ptr else None,
                                      int(bool(hydrostatic)), ctypes.byref(opts), ctypes.c_void_p(model_out_ptr),
                                      ctypes.c_void_p(chi2_ptr), ctypes.c_void_p(iters_ptr),
                                      ctypes.c_void_p(syn_ptr) if syn_ptr else None,
                                      ctypes.c_void_p(status_ptr) if status_ptr else None,
                                      ctypes.c_void_p(stream) if stream else None))

    def lm_perturbation(self, jac, diff, lam, svdtol=1e-4, reg_pen=None, reg_hss=None, dtype=1):
        """Batched GET_PERTURBATION: jac (npix, np, nfreq) normalised Jacobian
        -- float64 (IJACOBIAN, fz_lm_perturbation) or float32
        (fz_lm_perturbation_f32) --, diff (npix, nfreq), lam (npix,); optional
        reg_pen (npix, np) and reg_hss (npix, np, np); dtype 1 SVD, 2
        conjugate gradients.  Returns delta (npix, np)."""
        j = np.asarray(jac)
        j = np.ascontiguousarray(j, dtype=np.float32 if j.dtype == np.float32 else np.float64)
        d = np.ascontiguousarray(diff, dtype=np.float64)
        lm = np.ascontiguousarray(lam, dtype=np.float64)
        npix, npar, nf = j.shape
        rp = None if reg_pen is None else np.ascontiguousarray(reg_pen, dtype=np.float64).reshape(npix, npar)
        rh = None if reg_hss is None else np.ascontiguousarray(reg_hss, dtype=np.float64).reshape(npix, npar, npar)
        out = np.zeros((npix, npar))
        fn = lib().fz_lm_perturbation_f32 if j.dtype == np.float32 else lib().fz_lm_perturbation
        _check(fn(self._h, npix, npar, nf, _p(j), _p(d), _p(lm), None if rp is None else _p(rp),
                  None if rh is None else _p(rh), int(dtype), float(svdtol), _p(out)))
        return out

    def lm_rearange(self, models, delta, node_expansion=1):
        """Batched REARANGE_DA_MODEL: the normalised node perturbation delta
        (npix, np) applied to models (npix, 13, nz) with the node layout of
        rf_nodes(); returns the new models."""
        m = np.array(models, dtype=np.float32, order="C", copy=True)
        d = np.ascontiguousarray(delta, dtype=np.float64)
        if m.ndim != 3 or m.shape[1:] != (13, self.nz) or d.shape[0] != m.shape[0]:
            raise ValueError("models must be (npix, 13, nz) and delta (npix, np)")
        _check(lib().fz_lm_rearange(self._h, m.shape[0], _p(m), _p(d), int(node_expansion)))
        return m

    def forward_rf_device(self, model_ptr, ncol, syn_ptr, jac_ptr, model_out_ptr, status_ptr=0, stream=0,
                          hydrostatic=False):
        """Enqueue synthesis + node Jacobian on device pointers."""
        _check(lib().fz_forward_rf_device(self._h, int(ncol), ctypes.c_void_p(model_ptr), int(bool(hydrostatic)),
                                          ctypes.c_void_p(syn_ptr), ctypes.c_void_p(jac_ptr),
                                          ctypes.c_void_p(model_out_ptr),
                                          ctypes.c_void_p(status_ptr) if status_ptr else None,
                                          ctypes.c_void_p(stream) if stream else None))

    def forward_device(self, model_ptr, ncol, syn_ptr, model_out_ptr, status_ptr=0, stream=0, hydrostatic=False):
        """Enqueue a synthesis on device pointers (e.g. torch ``data_ptr()``)."""
        _check(lib().fz_forward_device(self._h, int(ncol), ctypes.c_void_p(model_ptr), he_mode(hydrostatic),
                                       ctypes.c_void_p(syn_ptr), ctypes.c_void_p(model_out_ptr),
                                       ctypes.c_void_p(status_ptr) if status_ptr else None,
                                       ctypes.c_void_p(stream) if stream else None))


def measure_fp64_peak(device=0):
    """Measured FP64 FMA peak of the device in TFLOP/s."""
    t = np.zeros(1)
    _check(lib().fz_measure_fp64_peak(int(device), _p(t)))
    return float(t[0])


def lm_update_lambda(chicur, chipre, lam, steps, precyc):
    """Batched UPDATE_LAMBDA on the GPU; returns the updated (chipre, lambda,
    steps, precyc) arrays."""
    cc = np.ascontiguousarray(chicur, dtype=np.float64)
    out = [np.array(a, dtype=np.float64, copy=True).reshape(cc.shape) for a in (chipre, lam, steps, precyc)]
    _check(lib().fz_lm_update_lambda(cc.size, _p(cc), *[_p(a) for a in out]))
    return tuple(out)


def rte_solve(eta, src, zz, bnd=None):
    """Formal solution on given absorption matrices (SET_BOUNDARY +
    OLD_ANALYTICAL_SOLVER): eta (ncol, nz, 7, nw) ETAI..RHOV [cm^-1], src
    (ncol, nz, nw), zz (nz,) km, bnd (ncol, nz) or None.  Returns SYN1D as
    (ncol, nw, 4) float64."""
    e = np.ascontiguousarray(eta, dtype=np.float32)
    ncol, nz, _, nw = e.shape
    s = np.ascontiguousarray(src, dtype=np.float32).reshape(ncol, nz, nw)
    z = np.ascontiguousarray(zz, dtype=np.float64)
    b = None if bnd is None else np.ascontiguousarray(bnd, dtype=np.int32).reshape(ncol, nz)
    out = np.zeros((ncol, nw, 4))
    _check(lib().fz_rte_solve(ncol, nz, nw, _p(e), _p(s), _p(z), None if b is None else _p(b), _p(out)))
    return out


def voigt(a, v):
    """The library's FP32 H(a, v), F(a, v) on the GPU (a, v broadcast)."""
    a, v = np.broadcast_arrays(np.asarray(a, dtype=np.float32), np.asarray(v, dtype=np.float32))
    a, v = np.ascontiguousarray(a).ravel(), np.ascontiguousarray(v).ravel()
    h, f = np.zeros_like(v), np.zeros_like(v)
    _check(lib().fz_voigt(v.size, _p(a), _p(v), _p(h), _p(f)))
    return h, f


def measure_fp32_peak(device=0):
    """Measured FP32 FMA peak of the device in TFLOP/s."""
    t = np.zeros(1)
    _check(lib().fz_measure_fp32_peak(int(device), _p(t)))
    return float(t[0])


from . import atmos  # noqa: E402,F401
