"""Learned initial guess of the inversion.

No counterpart in the reference: its LM starts from the model given in the
control file (or from the Stokes-moment assists of SET_TAU,
src/invert3d.f90:492-727).  Here an MLP maps the observed Stokes vector
(4 x NUMW, GAIN-normalised) to the node values of the free parameters -- the
CONTRACT_VECTOR averages (src/get_dmodel.f90:861-880) of T, Bx, By, Bz and
v_z over the hat basis of GET_INT_COEFS -- and the predicted nodes, expanded
on the height grid (EXPAND_VECTOR), replace those rows of a default model.

The network is trained on (model, profile) pairs that the library's own GPU
forward solver synthesises from seeded atmospheres, with the library's BF16
kernels (fz_mlp_*).  Device buffers are torch tensors (memory and streams
only); every FLOP of training and inference runs in libfzb200.so.
"""
import ctypes

import numpy as np

from . import FzError, _check, _p, atmos, lib

# (reference parameter, model row) of the free parameters the network predicts
PARAM_ROWS = ((1, 0), (2, 1), (4, 5), (5, 6), (6, 7), (7, 10))


def _bind():
    L = lib()
    if getattr(L, "_mlp_bound", False):
        return L
    P = ctypes.c_void_p
    L.fz_mlp_create.argtypes = [ctypes.POINTER(P), ctypes.c_int, P, ctypes.c_ulonglong, ctypes.c_int]
    L.fz_mlp_destroy.argtypes = [P]
    L.fz_mlp_nparams.argtypes = [P]
    L.fz_mlp_nparams.restype = ctypes.c_longlong
    L.fz_mlp_get_params.argtypes = [P, P, ctypes.c_int]
    L.fz_mlp_set_params.argtypes = [P, P]
    L.fz_mlp_forward_device.argtypes = [P, ctypes.c_int, P, P, P]
    L.fz_mlp_grad_device.argtypes = [P, ctypes.c_int, P, P, P]
    L.fz_mlp_train_device.argtypes = [P, ctypes.c_int, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                      ctypes.c_ulonglong, P]
    L.fz_mlp_forward_obs_device.argtypes = [P, ctypes.c_int, P, P, P, P, P]
    L.fz_mlp_set_loss_weights.argtypes = [P, P, ctypes.c_int]
    L.fz_warm_start_device.argtypes = [P, P, ctypes.c_int, P, P, P, P, P]
    L.fz_invert_warm.argtypes = [P, P, P, P, ctypes.c_int, P, P, ctypes.c_int, P, P, P, P, P, P]
    L._mlp_bound = True
    return L


class MLP:
    """Fully connected network dims[0] -> ... -> dims[-1], GELU in between."""

    def __init__(self, dims=(896, 1024, 1024, 512, 13), seed=0, device=0):
        L = _bind()
        self.dims = tuple(int(d) for d in dims)
        d = np.array(self.dims, dtype=np.int32)
        h = ctypes.c_void_p()
        _check(L.fz_mlp_create(ctypes.byref(h), len(self.dims) - 1, _p(d), int(seed), int(device)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _bind().fz_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nparams(self):
        return int(_bind().fz_mlp_nparams(self._h))

    def get_params(self, grads=False):
        out = np.zeros(self.nparams, dtype=np.float32)
        _check(_bind().fz_mlp_get_params(self._h, _p(out), int(bool(grads))))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.nparams:
            raise ValueError("expected %d parameters" % self.nparams)
        _check(_bind().fz_mlp_set_params(self._h, _p(p)))

    def set_loss_weights(self, w=None):
        """Per-output weights of the training loss (None: all 1)."""
        if w is None:
            _check(_bind().fz_mlp_set_loss_weights(self._h, None, 0))
            return
        a = np.ascontiguousarray(w, dtype=np.float32)
        _check(_bind().fz_mlp_set_loss_weights(self._h, _p(a), int(a.size)))

    def forward_device(self, n, x_ptr, y_ptr, stream=0):
        _check(_bind().fz_mlp_forward_device(self._h, int(n), ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                             ctypes.c_void_p(stream) if stream else None))

    def grad_device(self, n, x_ptr, t_ptr):
        loss = ctypes.c_float()
        _check(_bind().fz_mlp_grad_device(self._h, int(n), ctypes.c_void_p(x_ptr), ctypes.c_void_p(t_ptr),
                                          ctypes.byref(loss)))
        return loss.value

    def train_device(self, n, x_ptr, t_ptr, batch=1024, epochs=1, lr=1e-3, seed=0):
        loss = ctypes.c_float()
        _check(_bind().fz_mlp_train_device(self._h, int(n), ctypes.c_void_p(x_ptr), ctypes.c_void_p(t_ptr),
                                           int(batch), int(epochs), float(lr), int(seed), ctypes.byref(loss)))
        return loss.value


def hat_coefs(nz, nj):
    """GET_INT_COEFS (src/get_dmodel.f90:563-644): (nz, nj) hat functions."""
    c = np.zeros((nz, nj))
    if nj == 1:
        c[:, 0] = 1.0
        return c
    if nj == nz:
        return np.eye(nz)
    step = (nz - 1) / (nj - 1)
    pos = np.arange(nj) * step + 1.0
    i = np.arange(1, nz + 1, dtype=np.float64)
    for j in range(nj):
        ji, jf, jm = pos[max(j - 1, 0)], pos[min(j + 1, nj - 1)], pos[j]
        up = (i >= ji) & (i < jm)
        dn = (i > jm) & (i <= jf)
        c[up, j] = (i[up] - ji) / (jm - ji)
        c[dn, j] = (jf - i[dn]) / (jf - jm)
        c[i == jm, j] = 1.0
    return c


def default_models(npix, nz, b=100.0, seed=0):
    """The plain initial guess: the mean temperature stratification, its
    hydrostatic pressure, a field of (b, b, b) G and v_z = 0."""
    z = atmos.z_grid(nz)
    T = atmos.mean_temperature(z)[None, :]
    m = np.zeros((npix, 13, nz), dtype=np.float32)
    m[:, 0] = T
    m[:, 1] = atmos.hydrostatic_pg(T, z)
    m[:, 5:8] = b
    m[:, 12] = z[None, :]
    return m


class WarmStart:
    """Stokes vector -> node values -> initial model, for the node layout
    {reference parameter: NJ} of the inversion (T, Bx, By, Bz, v_z)."""

    def __init__(self, nz, nodes, numw, hidden=(1024, 1024, 512), seed=0, device=0):
        self.nz, self.numw = int(nz), int(numw)
        self.nodes = {int(p): int(n) for p, n in nodes.items() if n > 0}
        self.params = [(p, r) for p, r in PARAM_ROWS if p in self.nodes]
        self.nout = sum(self.nodes[p] for p, _ in self.params)
        self.coefs = {p: hat_coefs(self.nz, self.nodes[p]) for p, _ in self.params}
        self.mlp = MLP((4 * self.numw,) + tuple(hidden) + (self.nout,), seed=seed, device=device)
        self.xmu = self.xsd = self.tmu = self.tsd = None

    def targets(self, models):
        """Node values (CONTRACT_VECTOR) of models (n, 13, nz) -> (n, nout)."""
        cols = []
        for p, row in self.params:
            c = self.coefs[p]
            cols.append((models[:, row].astype(np.float64) @ c) / c.sum(axis=0))
        return np.concatenate(cols, axis=1)

    def expand(self, nodes_v, base):
        """Copies of base moved to the predicted node values (n, nout): each
        free row becomes base + EXPAND_VECTOR(nodes - CONTRACT_VECTOR(base)),
        the way the inversion itself perturbs a model.  Expanding the node
        values directly would replace the row by a piecewise-linear curve
        through node averages, which misses a steep stratification (T) by up
        to a third of a node step at the ends even for exact nodes."""
        m = np.array(base, dtype=np.float32, copy=True)
        cb = self.targets(m)
        j = 0
        for p, row in self.params:
            nj = self.nodes[p]
            d = nodes_v[:, j:j + nj] - cb[:, j:j + nj]
            m[:, row] = (m[:, row].astype(np.float64) + d @ self.coefs[p].T).astype(np.float32)
            j += nj
        return m

    def make_training_set(self, synth, ncol, seed, noise=1e-3, chunk=65536, bmax=2500.0):
        """Seeded atmospheres (|B| up to bmax G) synthesised on the GPU
        (hydrostatic) plus Gaussian noise: returns device tensors (x (ncol,
        4 numw), t (ncol, nout)) normalised with the set's own mean and
        spread."""
        import torch
        x = torch.empty((ncol, 4 * self.numw), dtype=torch.float32, device="cuda")
        t = np.empty((ncol, self.nout))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(int(seed) + 7)
        stream = torch.cuda.current_stream().cuda_stream
        for i in range(0, ncol, chunk):
            n = min(chunk, ncol - i)
            m = torch.from_numpy(atmos.make_columns(n, self.nz, seed=int(seed) * 1000003 + i, bmax=bmax)).cuda()
            syn = torch.empty((n, 4, self.numw), dtype=torch.float64, device="cuda")
            mo = torch.empty_like(m)
            synth.forward_device(m.data_ptr(), n, syn.data_ptr(), mo.data_ptr(), 0, stream=stream, hydrostatic=True)
            x[i:i + n] = (syn.reshape(n, -1) + noise * torch.randn(syn.reshape(n, -1).shape, device="cuda",
                                                                     dtype=torch.float64, generator=gen)).float()
            t[i:i + n] = self.targets(mo.cpu().numpy())
        self.xmu = x.mean(dim=0, keepdim=True)
        self.xsd = x.std(dim=0, keepdim=True) + 1e-6
        x.sub_(self.xmu).div_(self.xsd)
        self.tmu = t.mean(axis=0, keepdims=True)
        self.tsd = t.std(axis=0, keepdims=True) + 1e-12
        tt = torch.from_numpy(((t - self.tmu) / self.tsd).astype(np.float32)).cuda()
        return x, tt

    def _basis(self, dev):
        """Per free parameter, as FP64 tensors on dev: EXPAND (nj, nz), the
        hat averages of CONTRACT (nz, nj) and the least-squares inverse of
        EXPAND (nz, nj)."""
        import torch
        key = str(dev)
        cache = getattr(self, "_basis_cache", {})
        if key not in cache:
            b = {}
            for p, _ in self.params:
                c = self.coefs[p]
                b[p] = (torch.from_numpy(c.T.copy()).to(dev, torch.float64),
                        torch.from_numpy(c / c.sum(axis=0)).to(dev, torch.float64),
                        torch.from_numpy(np.linalg.pinv(c).T.copy()).to(dev, torch.float64))
            cache[key] = b
            self._basis_cache = cache
        return cache[key]

    def expand_nodes(self, nodes, base):
        """Tensor form of expand(): nodes (n, nout) FP64, base one MODEL
        (13, nz) float32 -> (n, 13, nz) float32 models, each free row
        base + EXPAND(nodes - CONTRACT(base)) (on the tensors' device)."""
        import torch
        basis = self._basis(nodes.device)
        m = base.expand(nodes.shape[0], -1, -1).clone()
        j = 0
        for p, row in self.params:
            nj = self.nodes[p]
            ct, cavg, _ = basis[p]
            b = base[row].to(torch.float64)
            m[:, row] = (b + (nodes[:, j:j + nj] - b @ cavg) @ ct).float()
            j += nj
        return m

    def fit_nodes(self, models, base):
        """Node values whose expansion on base (expand_nodes) reproduces the
        free rows of models (n, 13, nz) best, in the least-squares sense:
        CONTRACT(base) + EXPAND^+ (row - base row).  Exact (up to rounding)
        for models that differ from base by an expansion, as the
        inversion's models do."""
        import torch
        basis = self._basis(models.device)
        out = torch.empty((models.shape[0], self.nout), dtype=torch.float64, device=models.device)
        j = 0
        for p, row in self.params:
            nj = self.nodes[p]
            _, cavg, pinv = basis[p]
            b = base[row].to(torch.float64)
            out[:, j:j + nj] = b @ cavg + (models[:, row].to(torch.float64) - b) @ pinv
            j += nj
        return out

    def refine_targets(self, synth, x, t, opts, chunk=131072, stream=0):
        """LM-refined training targets.  Each training pixel is inverted
        (synth.invert_device with opts, hydrostatic) from the model of its
        true node values on the default guess, and its target becomes the
        node values whose expansion reproduces the inversion's best model
        (fit_nodes).  The true node averages of an atmosphere are not its
        best fit in the node space: the contraction averages away
        stratification the lines see and the expansion puts it back smeared,
        so their models sit well above the chi2 the inversion reaches next to
        them.  A network trained on the refined values learns the map from
        Stokes vectors to best-fit nodes, which is what a warm start needs.
        x, t: the standardised device training set of make_training_set;
        synth's node layout (rf_nodes) must be the network's.  The node
        normalisation is recomputed.  Returns the new standardised targets
        (device) and the inversion's statistics."""
        import time
        import torch
        if self.tsd is None:
            raise FzError("the network has no normalisation: make the training set first")
        t0 = time.perf_counter()
        dev = x.device
        ntot = x.shape[0]
        f64 = torch.float64
        tsd = torch.from_numpy(np.ravel(self.tsd)).to(dev, f64)
        tmu = torch.from_numpy(np.ravel(self.tmu)).to(dev, f64)
        xsd, xmu = self.xsd.to(f64), self.xmu.to(f64)
        base = torch.from_numpy(default_models(1, self.nz)[0]).to(dev)
        refined = torch.empty((ntot, self.nout), dtype=f64, device=dev)
        chis, its = [], []
        for i in range(0, ntot, chunk):
            n = min(chunk, ntot - i)
            start = self.expand_nodes(t[i:i + n].to(f64) * tsd + tmu, base)
            obs = (x[i:i + n].to(f64) * xsd + xmu).contiguous()
            out = torch.empty_like(start)
            chi = torch.empty(n, dtype=f64, device=dev)
            it = torch.empty(n, dtype=torch.int32, device=dev)
            st = torch.empty(n, dtype=torch.int32, device=dev)
            synth.invert_device(n, obs.data_ptr(), start.data_ptr(), out.data_ptr(), chi.data_ptr(), it.data_ptr(),
                                st.data_ptr(), hydrostatic=True, opts=opts, stream=stream)
            torch.cuda.synchronize()
            refined[i:i + n] = self.fit_nodes(out, base)
            chis.append(chi)
            its.append(it)
        r = refined.cpu().numpy()
        self.tmu = r.mean(axis=0, keepdims=True)
        self.tsd = r.std(axis=0, keepdims=True) + 1e-12
        tt = torch.from_numpy(((r - self.tmu) / self.tsd).astype(np.float32)).to(dev)
        chi = torch.cat(chis)
        info = {"pixels": int(ntot), "seconds": time.perf_counter() - t0,
                "mean_iterations": float(torch.cat(its).float().mean()), "median_chi2": float(torch.median(chi))}
        return tt, info

    def chi2_weights(self, synth, ncol=8192, seed=97, bmax=2500.0):
        """Loss weights under which the network's squared error approximates,
        to first order, the chi2 its prior costs: w_j = tsd_j^2 (J^T J)_jj
        (the node Jacobian of ncol seeded atmospheres of the training
        generator, mean over columns; tsd_j the spread of node j in the
        training set), normalised to mean 1.  Call after make_training_set,
        with synth's node layout the network's."""
        import torch
        if self.tsd is None:
            raise FzError("the network has no normalisation: make the training set first")
        stream = torch.cuda.current_stream().cuda_stream
        m = torch.from_numpy(atmos.make_columns(ncol, self.nz, seed=int(seed), bmax=bmax)).cuda()
        syn = torch.empty((ncol, 4, self.numw), dtype=torch.float64, device="cuda")
        jac = torch.empty((ncol, self.nout, 4 * self.numw), dtype=torch.float32, device="cuda")
        mo = torch.empty_like(m)
        synth.forward_rf_device(m.data_ptr(), ncol, syn.data_ptr(), jac.data_ptr(), mo.data_ptr(), 0, stream=stream,
                                hydrostatic=True)
        torch.cuda.synchronize()
        jj = (jac.double() ** 2).sum(dim=2).mean(dim=0).cpu().numpy()   # (J^T J)_jj, node order
        # the network's outputs follow PARAM_ROWS, the Jacobian's columns the
        # reference's parameter order: the same sequence for this layout
        w = jj * np.ravel(self.tsd) ** 2
        return (w / w.mean()).astype(np.float32)

    def fit(self, x, t, epochs=8, batch=1024, lr=1e-3, seed=0, loss_weights=None):
        """Adam on the device training set; returns the last epoch's mean loss.
        loss_weights: per-output weights of the squared error (e.g.
        chi2_weights), None for the plain mean squared error."""
        self.mlp.set_loss_weights(loss_weights)
        import torch
        torch.cuda.synchronize()
        n = (x.shape[0] // batch) * batch
        return self.mlp.train_device(n, x.data_ptr(), t.data_ptr(), batch=batch, epochs=epochs, lr=lr, seed=seed)

    def predict_nodes(self, obs):
        """obs (npix, 4, numw) -> node values (npix, nout) in physical units."""
        import torch
        if self.xmu is None:
            raise FzError("the network has no normalisation: train it first")
        x = torch.from_numpy(np.ascontiguousarray(obs, dtype=np.float32).reshape(obs.shape[0], -1)).cuda()
        x = ((x - self.xmu) / self.xsd).contiguous()
        y = torch.empty((x.shape[0], self.nout), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        self.mlp.forward_device(x.shape[0], x.data_ptr(), y.data_ptr())
        return y.cpu().numpy().astype(np.float64) * self.tsd + self.tmu

    def norm(self):
        """The network's standardisation as the library takes it: FP32 input
        mean and spread (NFREQ each), node mean and spread (nout each)."""
        if self.xmu is None:
            raise FzError("the network has no normalisation: train it first")
        xm = self.xmu.detach().reshape(-1).float().cpu().numpy() if hasattr(self.xmu, "detach") else self.xmu
        xs = self.xsd.detach().reshape(-1).float().cpu().numpy() if hasattr(self.xsd, "detach") else self.xsd
        return np.concatenate([np.ravel(xm), np.ravel(xs), np.ravel(self.tmu), np.ravel(self.tsd)]).astype(np.float32)

    def models_device(self, synth, n, obs_ptr, base_ptr, out_ptr, stream=0):
        """Warm-start models on the device through fz_warm_start_device:
        obs_ptr (n, NFREQ) FP64 observations, base_ptr one MODEL(NZ,13)
        float32, out_ptr (n, 13, nz) float32; the node layout of synth
        (rf_nodes) must be the network's."""
        import torch
        if getattr(self, "_dnorm", None) is None:
            self._dnorm = torch.from_numpy(self.norm()).cuda()
        _check(_bind().fz_warm_start_device(synth._h, self.mlp._h, int(n), ctypes.c_void_p(obs_ptr),
                                            ctypes.c_void_p(self._dnorm.data_ptr()), ctypes.c_void_p(base_ptr),
                                            ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream) if stream else None))

    def initial_models_device(self, x_obs, base):
        """Warm-start models on the device: x_obs (npix, 4*numw) float32 raw
        Stokes (device tensor), base (npix, 13, nz) float32 device tensor whose
        free-parameter rows are replaced.  Returns a new device tensor."""
        import torch
        n = x_obs.shape[0]
        x = ((x_obs - self.xmu) / self.xsd).contiguous()
        y = torch.empty((n, self.nout), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        self.mlp.forward_device(n, x.data_ptr(), y.data_ptr())
        if not hasattr(self, "_dev"):
            self._dev = (torch.from_numpy(self.tsd.astype(np.float32)).cuda(),
                         torch.from_numpy(self.tmu.astype(np.float32)).cuda(),
                         {p: torch.from_numpy(self.coefs[p].T.astype(np.float32)).cuda() for p, _ in self.params},
                         {p: torch.from_numpy((self.coefs[p] / self.coefs[p].sum(axis=0)).astype(np.float32)).cuda()
                          for p, _ in self.params})
        tsd, tmu, ct, cavg = self._dev
        nodes_v = y * tsd + tmu
        m = base.clone()
        j = 0
        for p, row in self.params:
            nj = self.nodes[p]
            # base + EXPAND(nodes - CONTRACT(base)), as expand()
            m[:, row] = m[:, row] + (nodes_v[:, j:j + nj] - m[:, row] @ cavg[p]) @ ct[p]
            j += nj
        return m

    def initial_models(self, obs, base=None, out=None):
        """Warm-start models for host observations obs (npix, 4, numw): the
        network and the node expansion run on the device; returns host
        models (npix, 13, nz) float32, in out if given (e.g. pinned memory)
        (base: host models whose other rows are kept, default_models() if
        None)."""
        import torch
        n = obs.shape[0]
        x = torch.from_numpy(np.ascontiguousarray(obs).reshape(n, -1)).cuda().float()
        if base is None:
            b = torch.from_numpy(default_models(1, self.nz)).cuda().expand(n, -1, -1)
        else:
            b = torch.from_numpy(np.ascontiguousarray(base, dtype=np.float32)).cuda()
        m = self.initial_models_device(x, b)
        if out is None:
            return m.cpu().numpy()
        if out.shape != (n, 13, self.nz) or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float32 (npix, 13, nz) array")
        torch.from_numpy(out).copy_(m)
        return out
