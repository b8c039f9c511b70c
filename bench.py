#!/usr/bin/env python3
"""Benchmark of the FIRTEZ-dz hot path on B200: batched pixel-wise LM
inversion with the learned warm start, against LM from the default guess.

Workload (one GPU): a seeded 512 x 512 field of model atmospheres, 128 heights
from -0.5 to +1.5 Mm, Fe I 6301.5 + 6302.5 x 112 wavelengths at 21.5 mA
(NUMW = 224, NFREQ = 896), observations = the GPU synthesis (hydrostatic) of
the field plus Gaussian noise of 1e-3 Ic.  Free parameters on nodes: T 5,
Bx, By, Bz, v_z 2 each (NP = 13).  Plain stop rule per pixel: the
reference's STEPS > MAXSTEPS (5), an accepted step gaining less than 1e-3 in
chi2 (relative), or 40 iterations.  The warm start is the MLP
896-1024-1024-512-13 (GELU), trained before the timed region with the
library's BF16 tcgen05 kernels on pairs the GPU forward solver synthesises
from seeded atmospheres (1M by default), its targets the node values of an
LM inversion of each training pixel started from its true node values
(WarmStart.refine_targets; --refine-steps 0: the true node averages).

Calibration, before the timed region: plain LM from the default guess on
32,768 pixels of a separate seeded set (same generator, same noise); the
acceptance level T is the 20th percentile of their chi2 (--accept-quantile).

One step = the inversion of the whole 512 x 512 field (one inversion call
of 262,144 pixels), inputs resident in HBM.  Headline arm (``value``): the
deployable NN-warm rule -- the network's model of every pixel is evaluated
once; a pixel whose chi2 there is at or below T is converged with it, every
other pixel restarts at once from the default guess in the same slot pool
and runs plain LM (fallback_steps -1, fallback_free).  ``value`` = its
pixels/s; the plain arm (LM from the default guess, plain stop rules; at
most --plain-steps timed steps) is the yardstick, and the line gives the speed-up over it, both median chi2, the
fraction of pixels whose chi2 ends above 1.1x their plain-LM chi2 and the
parameter errors against the true atmospheres.  Beside it (--sub-steps
steps each): the same rule at two other quantiles, NN-warm LM with the plain
stop rules only, and plain LM from SET_TAU's assisted guess.  ``e2e``: the headline arm through
fz_invert_warm from pinned host memory.  Multi-GPU: each rank inverts tiles of
its own field (weak scaling, no collective on the data path; a barrier and the
max over ranks of each time).

``roofline``: the dominant kernel of the headline arm against the pipe that
bounds it (FP32 or FP64 FLOP per column counted by ncu on 2048 columns of
this workload, profiles/flops.json, over the peak of an FMA-chain kernel
measured in the same run), DRAM traffic per launch from ncu and the HBM
fraction as side figures.

``--impl reference`` times the CPU restatement of the reference (oracle/: the
Fortran reference cannot be built on this image, no gfortran/MPI/LAPACK),
LM from the default guess, on bounded pixel samples with all host cores.
``--probe-kernels N`` runs one synthesis and one node-Jacobian call on N
columns of the workload twice and exits (the launches ncu counts FLOPs on);
``--flops-from CSV`` turns that ncu CSV into profiles/flops.json.
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "firtez-dz_b200")
METRIC = "converged pixels/s at plain-LM χ² (NN-warm vs plain, 1 B200); synth columns·λ/s"
UNIT = "pixels/s"
NODES = {1: 5, 4: 2, 5: 2, 6: 2, 7: 2}


class Ranks:
    """The bench's process group (one process per GPU, weak scaling): a
    barrier and the maximum over ranks of a time; NCCL on the GPUs, gloo in
    the CPU tests.  world == 1: no process group."""

    def __init__(self, world, backend="nccl", device="cuda", timeout_s=300):
        self.world, self.device, self.dist = world, device, None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def maxms(self, ms):
        if self.dist is None:
            return ms
        import torch
        t = torch.tensor([float(ms)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def field_seed(rank, chunk):
    """Seed of the field's chunk of seeded atmospheres on one rank: every
    rank inverts a field of its own."""
    return 777000 + 1000 * rank + chunk


def load_package():
    name = "firtez_dz_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index, tag):
        self.index = index
        self.proc = None
        # the raw samples go to $FZ_CLOCKS_DIR (default: the system's temporary directory)
        import tempfile
        self.path = os.path.join(os.environ.get("FZ_CLOCKS_DIR", tempfile.gettempdir()),
                                 "clocks_%s_rank%d.csv" % (tag, index))

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def _oracle_side():
    """The modules the CPU arms use: the oracle's ctypes wrapper (tests/orc.py),
    its LM (oracle/lm_oracle.py) and the workload generator atmos.py loaded as
    a plain module -- never the package or libfzb200.so."""
    for d in (os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")):
        if d not in sys.path:
            sys.path.insert(0, d)
    import orc
    import lm_oracle as lmo
    name = "fz_workload_atmos"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "atmos.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules[name] = mod
    return orc, lmo, sys.modules[name]


def cpu_workload():
    """Line table and regions of the workload parsed by the oracle."""
    orc, _, atm = _oracle_side()
    lines = orc.parse_lines(atm.line_database_text())
    return lines, orc.regions(atm.lines_section(2), lines)


def default_guess(atm, npix, nz, b=100.0):
    """The plain initial guess: the mean temperature stratification, its
    hydrostatic pressure, a field of (b, b, b) G and v_z = 0."""
    z = atm.z_grid(nz)
    T = atm.mean_temperature(z)[None, :]
    m = np.zeros((npix, 13, nz), dtype=np.float32)
    m[:, 0] = T
    m[:, 1] = atm.hydrostatic_pg(T, z)
    m[:, 5:8] = b
    m[:, 12] = z[None, :]
    return m


def cpu_lm_sample(lines, reg, he, nz, npix, seed, nthreads=0):
    """The oracle's pixel-wise LM (plain initial guess) on npix pixels of the
    workload, OpenMP over the pixels of each forward pass; returns (pixels/s,
    seconds, median chi2)."""
    orc, lmo, atm = _oracle_side()
    gain, _ = orc.gain(lines, reg)
    true = atm.make_columns(npix, nz, seed=seed)
    obs, _, _ = orc.forward(lines, reg, gain, true, hydrostatic=he, nthreads=nthreads)
    obs = obs.reshape(npix, -1) + np.random.default_rng(seed).normal(0.0, 1e-3, (npix, obs.shape[1] * obs.shape[2]))
    init = default_guess(atm, npix, nz)
    w = lmo.weights(obs.shape[1] // 4, isigma=1e-3)

    def fwd(models):
        syn, jac, mo, st = orc.forward_rf(lines, reg, gain, models, NODES, hydrostatic=he, nthreads=nthreads)
        return syn.reshape(len(models), -1), np.transpose(jac, (0, 2, 1)), mo, st

    t0 = time.perf_counter()
    _, chi, _ = lmo.invert(fwd, obs, init, NODES, w, maxsteps=5, maxit=40, dchi2=1e-3)
    el = time.perf_counter() - t0
    return npix / el, el, float(np.median(chi))


def cpu_synth_sample(lines, reg, he, nz, ncol, seed, nthreads=0):
    """The oracle's FP64 synthesis of ncol seeded columns, OpenMP over
    columns; returns (columns*lambda/s, seconds)."""
    orc, _, atm = _oracle_side()
    gain, _ = orc.gain(lines, reg)
    m = atm.make_columns(ncol, nz, seed=seed)
    numw = int(reg["numwave"].sum())
    t0 = time.perf_counter()
    orc.forward(lines, reg, gain, m, hydrostatic=he, nthreads=nthreads)
    el = time.perf_counter() - t0
    return ncol * numw / el, el


PROBE_SEED = 3
CALIB_SEED = 909090
C5_SEED = 5050


SAHA_MAX_COLS = 1024   # batches up to this size run the chain on k_saha's precomputed Saha factors


def probe_kernels(fz, lines, reg, nz, n):
    """One synthesis and one node-Jacobian call (fz_forward_device,
    fz_forward_rf_device) on n seeded columns of the workload, twice: every
    launch processes all n columns, for per-opcode counts under ncu."""
    import torch
    ctx = fz.Synthesis(lines, reg, nz=nz)
    ctx.rf_nodes(NODES)
    m = torch.from_numpy(fz.atmos.make_columns(n, nz, seed=PROBE_SEED)).cuda()
    syn = torch.empty((n, 4, ctx.numw), dtype=torch.float64, device="cuda")
    jac = torch.empty((n, sum(NODES.values()), 4 * ctx.numw), dtype=torch.float32, device="cuda")
    mo = torch.empty_like(m)
    for _ in range(2):
        ctx.forward_device(m.data_ptr(), n, syn.data_ptr(), mo.data_ptr(), 0, hydrostatic=True)
        ctx.forward_rf_device(m.data_ptr(), n, syn.data_ptr(), jac.data_ptr(), mo.data_ptr(), 0, hydrostatic=True)
    torch.cuda.synchronize()
    print(json.dumps({"probe_columns": n, "nz": nz, "numw": ctx.numw, "mean_I": float(syn[:, 0].mean())}))


def flops_table(csv_path, ncol, nz, numw, out_path):
    """FLOP per column of each kernel from an ncu CSV of --probe-kernels
    (metrics smsp__sass_thread_inst_executed_op_{ffma,fadd,fmul,dfma,dadd,
    dmul}_pred_on.sum): FP32 = 2 ffma + fadd + fmul, FP64 likewise, per
    launch over its ncol columns; the median over a kernel's launches.  A
    kernel is bound by the pipe with more FLOP."""
    import csv
    import re
    rows = [r for r in csv.reader(open(csv_path)) if r]
    h = next(i for i, r in enumerate(rows) if r[0] == "ID")
    hdr = rows[h]
    per = {}
    for r in rows[h + 1:]:
        rec = dict(zip(hdr, r))
        name = re.search(r"(k_\w+)", rec["Kernel Name"]).group(1)
        v = float(rec["Metric Value"].replace(",", ""))
        per.setdefault((rec["ID"], name), {})[rec["Metric Name"]] = v
    acc = {}
    for (_, name), m in per.items():
        g = lambda op: m.get("smsp__sass_thread_inst_executed_op_%s_pred_on.sum" % op, 0.0)  # noqa: E731
        f32 = 2 * g("ffma") + g("fadd") + g("fmul")
        f64 = 2 * g("dfma") + g("dadd") + g("dmul")
        acc.setdefault(name, []).append((f32 / ncol, f64 / ncol, m.get("gpu__time_duration.sum", 0.0)))
    kern = {}
    for name, v in acc.items():
        v = sorted(v)
        f32, f64, _ = v[len(v) // 2]
        pipe = "fp64" if f64 > f32 else "fp32"
        kern[name] = {"pipe": pipe, "flop_per_column": f64 if pipe == "fp64" else f32,
                      "fp32_flop_per_column": f32, "fp64_flop_per_column": f64,
                      "flop_per_column_height_lambda": (f64 if pipe == "fp64" else f32) / (nz * numw),
                      "launches": len(v)}
    doc = {"_comment": "FLOP per column counted by ncu (thread-level ffma/fadd/fmul and dfma/dadd/dmul, an FMA "
                       "counted as 2) on --probe-kernels %d: %d seeded columns, NZ %d, NUMW %d, hydrostatic, nodes "
                       "T5 Bx2 By2 Bz2 vz2; bench.py multiplies by the columns of a launch" % (ncol, ncol, nz, numw),
           "kernels": kern}
    old = json.load(open(out_path)) if os.path.exists(out_path) else {"_comment": "", "kernels": {}}
    if "k_saha" in kern:
        # a small batch (at most SAHA_MAX_COLS columns) runs the chain on
        # precomputed Saha factors: its two kernels join the table of the
        # full-batch probe
        doc = old
        doc["kernels"].update({"k_saha": kern["k_saha"], "k_chain_pre": kern["k_chain"]})
        doc["_comment_small"] = ("k_saha and k_chain_pre (the chain of a batch of at most %d columns on precomputed "
                                 "Saha factors) from --probe-kernels %d" % (SAHA_MAX_COLS, ncol))
    else:
        # a full-batch table keeps the small-batch kernels of an earlier probe
        for k in ("k_saha", "k_chain_pre"):
            if k in old.get("kernels", {}):
                doc["kernels"][k] = old["kernels"][k]
        if "_comment_small" in old:
            doc["_comment_small"] = old["_comment_small"]
    with open(out_path, "w") as f:
        json.dump(doc, f, indent=1)
    print(json.dumps(doc))


TARGETS = ("LM-refined node values: each training pixel inverted from its true node values (MAXSTEPS 2, "
           "at most 15 iterations), the target the nodes of the best model")


def refine_opts(fz, a):
    """Stop rules of the inversion that refines the training targets."""
    return fz.LMOpts(maxsteps=a.refine_steps, maxit=15, dchi2=1e-3, isigma=1e-3, slots=65536)


def c5_sub_metric(a, fz, rank, world, stream, maxms):
    """The large multi-line workload: columns of a 1024 x 1024 field x 160
    heights, Fe I 6301.5, 6302.5, 15648.5 and 15652.9 x 96 wavelengths each
    (NUMW 384, NFREQ 1536), |B| up to 4000 G, noise 1e-3 Ic.  Its own network
    (MLP 1536-1024-1024-512-13) trained on --c5-train-pairs pairs, its own
    calibration (plain LM on 16,384 pixels, T at --accept-quantile), then the
    deployable NN-warm rule against plain LM on --c5-tiles tiles of 65,536
    pixels of the field (one warm-up step each, CUDA events, the max over
    ranks)."""
    import torch
    from firtez_dz_b200 import warmstart as ws
    nz, tile = 160, 65536
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(4), lines)
    ctx = fz.Synthesis(lines, reg, nz=nz, device=torch.cuda.current_device())
    numw = ctx.numw
    nf = 4 * numw
    npx = tile * a.c5_tiles
    t0 = time.perf_counter()
    obs = torch.empty((npx, nf), dtype=torch.float64, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(5151 + rank)
    for i in range(0, npx, tile):
        m = torch.from_numpy(fz.atmos.make_columns(tile, nz, seed=C5_SEED + 1000 * rank + i // tile,
                                                   bmax=4000.0)).cuda()
        syn = torch.empty((tile, 4, numw), dtype=torch.float64, device="cuda")
        mo = torch.empty_like(m)
        ctx.forward_device(m.data_ptr(), tile, syn.data_ptr(), mo.data_ptr(), 0, stream=stream, hydrostatic=True)
        obs[i:i + tile] = syn.reshape(tile, nf) + 1e-3 * torch.randn((tile, nf), dtype=torch.float64,
                                                                     device="cuda", generator=gen)
    del m, syn, mo
    warm = ws.WarmStart(nz, NODES, numw, seed=11 + rank)
    x, t = warm.make_training_set(ctx, a.c5_train_pairs, seed=61 + rank, noise=1e-3, bmax=4000.0)
    ctx.rf_nodes(NODES)
    refine = None
    if a.refine_steps > 0:
        t, refine = warm.refine_targets(ctx, x, t, refine_opts(fz, a), stream=stream)
    loss = warm.fit(x, t, epochs=a.c5_epochs, batch=1024, lr=1e-3, seed=1)
    del x, t
    torch.cuda.empty_cache()
    t_train = time.perf_counter() - t0
    base = torch.from_numpy(ws.default_models(tile, nz)).cuda()
    base1 = base[0].contiguous()
    init = torch.empty_like(base)
    out = torch.empty_like(base)
    chi = torch.empty(tile, dtype=torch.float64, device="cuda")
    it = torch.empty(tile, dtype=torch.int32, device="cuda")
    st = torch.empty(tile, dtype=torch.int32, device="cuda")
    slots = min(16384, tile)
    opts = fz.LMOpts(maxsteps=5, maxit=40, dchi2=1e-3, isigma=1e-3, slots=slots)
    # calibration on a separate seeded set
    ncal = 16384
    cm = torch.from_numpy(fz.atmos.make_columns(ncal, nz, seed=C5_SEED + 777, bmax=4000.0)).cuda()
    cs = torch.empty((ncal, 4, numw), dtype=torch.float64, device="cuda")
    cmo = torch.empty_like(cm)
    ctx.forward_device(cm.data_ptr(), ncal, cs.data_ptr(), cmo.data_ptr(), 0, stream=stream, hydrostatic=True)
    cg = torch.Generator(device="cuda")
    cg.manual_seed(C5_SEED)
    cobs = cs.reshape(ncal, nf) + 1e-3 * torch.randn((ncal, nf), dtype=torch.float64, device="cuda", generator=cg)
    ctx.invert_device(ncal, cobs.data_ptr(), base.data_ptr(), out.data_ptr(), chi.data_ptr(), it.data_ptr(),
                      st.data_ptr(), hydrostatic=True, opts=opts, stream=stream)
    T = float(torch.quantile(chi[:ncal], a.accept_quantile))
    del cm, cs, cmo, cobs
    accept = torch.full((tile,), T, dtype=torch.float64, device="cuda")
    opts_nn = fz.LMOpts(maxsteps=5, maxit=40, dchi2=1e-3, isigma=1e-3, slots=slots, fallback=1.0,
                        fallback_model=base1.data_ptr(), fallback_steps=-1, fallback_free=True)
    res = {"plain": [], "nn": []}

    def run(arm, k, keep):
        o = obs[k * tile:(k + 1) * tile]
        if arm == "plain":
            ini = base
        else:
            ini = init
            warm.models_device(ctx, tile, o.data_ptr(), base1.data_ptr(), ini.data_ptr(), stream=stream)
        ctx.invert_device(tile, o.data_ptr(), ini.data_ptr(), out.data_ptr(), chi.data_ptr(), it.data_ptr(),
                          st.data_ptr(), hydrostatic=True, opts=opts_nn if arm == "nn" else opts, stream=stream,
                          target_ptr=accept.data_ptr() if arm == "nn" else 0)
        if keep:
            res[arm].append((chi.cpu().numpy().copy(), it.cpu().numpy().copy(), int(st.max().item())))

    ms = {}
    for arm in ("plain", "nn"):
        run(arm, 0, False)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(a.c5_tiles):
            run(arm, k, True)
        e1.record()
        torch.cuda.synchronize()
        ms[arm] = maxms(e0.elapsed_time(e1) / a.c5_tiles)
    cp = np.concatenate([r[0] for r in res["plain"]])
    cn = np.concatenate([r[0] for r in res["nn"]])
    itp = np.concatenate([r[1] for r in res["plain"]])
    itn = np.concatenate([r[1] for r in res["nn"]])
    vp = world * tile / (ms["plain"] * 1e-3)
    vn = world * tile / (ms["nn"] * 1e-3)
    return {"value": vn, "unit": UNIT, "plain_value": vp, "speedup_vs_plain": vn / vp,
            "median_chi2": float(np.median(cn)), "median_chi2_plain": float(np.median(cp)),
            "mean_iterations": float(itn.mean()), "mean_iterations_plain": float(itp.mean()),
            "frac_pixels_chi2_above_1.1x_plain": float(np.mean(cn > 1.1 * cp)),
            "frac_pixels_restarted": float(np.mean(itn > 1)),
            "status_errors": max(r[2] for arm in res for r in res[arm]),
            "ms_per_step": ms["nn"], "ms_per_step_plain": ms["plain"], "T": T, "calibration_pixels": ncal,
            "mlp": {"layers": [nf, 1024, 1024, 512, 13], "train_pairs": a.c5_train_pairs, "epochs": a.c5_epochs,
                    "final_loss": loss, "field_and_training_s": t_train,
                    "targets": TARGETS if refine else "the true atmospheres' node averages", "refine": refine},
            "workload": "%d tiles of %d pixels of a seeded 1024x1024 field (rank %d's rows), %d heights, Fe I "
                        "6301.5, 6302.5, 15648.5, 15652.9 x 96 lambda (NUMW %d), |B| <= 4000 G, noise 1e-3 Ic, "
                        "nodes T5 Bx2 By2 Bz2 vz2; the headline's rule and stop rules, %d slots"
                        % (a.c5_tiles, tile, rank, nz, numw, slots)}


def reference_arm(a, config, he):
    """``--impl reference``: the CPU restatement of the reference (the Fortran
    reference cannot be built here: no gfortran/MPI/LAPACK) timed on all host
    cores -- plain LM from the default guess, each step a bounded sample of
    4 x cores pixels of the workload; beside it the FP64 synthesis of 256
    columns of the synthesis sub-metric's shape.  Rank 0 only."""
    lines, reg = cpu_workload()
    cores = os.cpu_count()
    npx = a.cpu_pixels if a.cpu_pixels > 0 else 4 * cores
    numw = int(reg["numwave"].sum())
    tot_t, chis = 0.0, []
    for i in range(a.warmup):
        cpu_lm_sample(lines, reg, he, a.nz, 2, seed=900 + i)
    for i in range(a.steps):
        _, el, c = cpu_lm_sample(lines, reg, he, a.nz, npx, seed=1000 + i)
        tot_t += el
        chis.append(c)
    value = float(a.steps * npx / tot_t)
    sv, sel = cpu_synth_sample(lines, reg, he, a.nz, 256, seed=2)
    sample = ("%d pixels per step (4 x %d cores), LM from the default guess to the plain stop rules, FP64 C++ "
              "restatement of the reference's forward/RF routines (OpenMP over pixels) + numpy/LAPACK LM; the "
              "Fortran reference needs gfortran/MPI/LAPACK, absent on this image" % (npx, cores))
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot_t / a.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": config, "median_chi2": float(np.median(chis)),
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
           "synthesis": {"value": sv, "unit": "columns*lambda/s", "seconds": sel,
                         "workload": "256 columns x %d heights x %d lambda, hydrostatic, FP64 oracle on %d cores"
                                     % (a.nz, numw, cores)},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--field", type=int, default=512, help="field side (pixels)")
    ap.add_argument("--tile", type=int, default=0, help="pixels per step (0: the whole field)")
    ap.add_argument("--slots", type=int, default=8192)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--train-pairs", type=int, default=1048576)
    ap.add_argument("--refine-steps", type=int, default=2,
                    help="MAXSTEPS of the LM that refines the training targets (0: the true node averages)")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--cpu-pixels", type=int, default=0, help="CPU LM pixels per sample (0: 4 x cores)")
    ap.add_argument("--synth-cols", type=int, default=256 * 256)
    ap.add_argument("--rf-chunk", type=int, default=4096, help="columns per full-height RF call")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--accept-quantile", type=float, default=0.2,
                    help="T = this quantile of the calibration set's plain-LM chi2")
    ap.add_argument("--calib-pixels", type=int, default=32768)
    ap.add_argument("--sub-steps", type=int, default=1, help="timed steps of each secondary arm (at most --steps)")
    ap.add_argument("--plain-steps", type=int, default=4, help="timed steps of the plain-LM yardstick (at most --steps)")
    ap.add_argument("--c5-tiles", type=int, default=2, help="65536-pixel tiles of the four-line workload (0: off)")
    ap.add_argument("--c5-train-pairs", type=int, default=524288)
    ap.add_argument("--c5-epochs", type=int, default=4)
    ap.add_argument("--probe-kernels", type=int, default=0, help="run the FLOP-count launches on N columns and exit")
    ap.add_argument("--flops-from", default="", help="ncu CSV of --probe-kernels -> profiles/flops.json, then exit")
    a = ap.parse_args()
    if a.tile <= 0 or a.tile > a.field * a.field:
        a.tile = a.field * a.field   # one inversion call per step over the whole field
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    he = True
    numw = 2 * 112
    nf = 4 * numw
    config = {"workload": "batched LM inversion, %dx%d pixels x %d heights, Fe I 6301.5+6302.5 x 112 lambda, "
                          "nodes T5 Bx2 By2 Bz2 vz2 (NP=13), noise 1e-3 Ic, NN-warm start "
                          "(MLP 896-1024-1024-512-13) vs default guess" % (a.field, a.field, a.nz),
              "pixels_per_gpu": a.field * a.field, "pixels_per_step": a.tile, "nz": a.nz, "numw": numw,
              "hydrostatic": he, "stop": "STEPS>5 | rel. dchi2<1e-3 on an accepted step | 40 iterations",
              "l2": "inputs larger than L2 (observations %.0f MB per GPU)" % (a.field * a.field * nf * 8 / 1e6),
              "parallelism": "pixel tiles sharded per GPU" if world > 1 else "single GPU"}

    if a.flops_from:
        flops_table(a.flops_from, a.probe_kernels or 2048, a.nz, numw, os.path.join(ROOT, "profiles", "flops.json"))
        return
    if a.impl == "reference":
        # before anything of the product is imported or loaded
        if rank == 0:
            reference_arm(a, config, he)
        return

    fz = load_package()
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    assert int(reg["numwave"].sum()) == numw
    if a.probe_kernels:
        probe_kernels(fz, lines, reg, a.nz, a.probe_kernels)
        return

    import torch
    from firtez_dz_b200 import warmstart as ws
    torch.cuda.set_device(local)
    ranks = Ranks(world)
    barrier, maxms = ranks.barrier, ranks.maxms

    ctx = fz.Synthesis(lines, reg, nz=a.nz, device=local)
    stream = torch.cuda.current_stream().cuda_stream
    # ---------------------------------------------------------------- field
    npix = a.field * a.field
    obs = torch.empty((npix, nf), dtype=torch.float64, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(4242 + rank)
    chunk = 65536
    warm = ws.WarmStart(a.nz, NODES, numw, seed=5 + rank)
    true_models = torch.empty((npix, 13, a.nz), dtype=torch.float32, device="cuda")
    for i in range(0, npix, chunk):
        n = min(chunk, npix - i)
        m = torch.from_numpy(fz.atmos.make_columns(n, a.nz, seed=field_seed(rank, i // chunk))).cuda()
        syn = torch.empty((n, 4, numw), dtype=torch.float64, device="cuda")
        mo = torch.empty_like(m)
        ctx.forward_device(m.data_ptr(), n, syn.data_ptr(), mo.data_ptr(), 0, stream=stream, hydrostatic=True)
        obs[i:i + n] = syn.reshape(n, nf) + 1e-3 * torch.randn((n, nf), dtype=torch.float64, device="cuda",
                                                               generator=gen)
        true_models[i:i + n] = mo
    base = torch.from_numpy(ws.default_models(a.tile, a.nz)).cuda()
    base1 = base[0].contiguous()                      # the one default model the warm start moves
    nn_init = torch.empty_like(base)
    # --------------------------------------------------------------- network
    t0 = time.perf_counter()
    x, t = warm.make_training_set(ctx, a.train_pairs, seed=31 + rank, noise=1e-3)
    t1 = time.perf_counter()
    ctx.rf_nodes(NODES)
    refine = None
    if a.refine_steps > 0:
        t, refine = warm.refine_targets(ctx, x, t, refine_opts(fz, a), stream=stream)
    t2 = time.perf_counter()
    loss = warm.fit(x, t, epochs=a.epochs, batch=1024, lr=1e-3, seed=1)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    del x, t
    torch.cuda.empty_cache()
    mlp_info = {"train_pairs": a.train_pairs, "epochs": a.epochs, "batch": 1024, "final_loss": loss,
                "targets": TARGETS if refine else "the true atmospheres' node averages",
                "refine": refine, "gen_s": t1 - t0, "refine_s": t2 - t1, "train_s": t3 - t2,
                "params": warm.mlp.nparams}
    opts = fz.LMOpts(maxsteps=5, maxit=40, dchi2=1e-3, isigma=1e-3, slots=a.slots)
    tuned = None
    if not a.no_tune:
        # the autotuner: launch shapes of the RF chemistry kernels on default-guess
        # columns, then the slot count by inverting the first tile (plain LM)
        # once per candidate; the arms below use the tuned slot count
        t0 = time.perf_counter()
        tf = ctx.autotune_forward(base.data_ptr(), min(8192, a.tile), hydrostatic=True)
        ntune = min(a.tile, 131072)   # the slot count on the field's first 131,072 pixels
        cands = tuple(c for c in (ntune // 4, ntune // 2, ntune) if c >= 256)
        tl = ctx.autotune_lm(ntune, obs[:ntune].data_ptr(), base.data_ptr(), candidates=cands, opts=opts)
        tuned = {"shapes": ctx.tune(), "slot_candidates": list(cands),
                 "forward_ms": {k: tf[k] for k in ("chain_ms", "chemder_ms", "opac_rf_ms")},
                 "lm_pixels_per_s_at_best": tl["lm_pixels_per_s"], "tuning_s": time.perf_counter() - t0}
        opts = fz.LMOpts(maxsteps=5, maxit=40, dchi2=1e-3, isigma=1e-3, slots=0)
    # ----------------------------------------------------------- calibration
    # plain LM from the default guess on a separate seeded set (same
    # generator, same noise; the same set on every rank): T = a quantile of
    # its chi2, the level at which a warm-start model is accepted
    t0 = time.perf_counter()
    ncal = min(a.calib_pixels, a.tile)
    cal_m = torch.from_numpy(fz.atmos.make_columns(ncal, a.nz, seed=CALIB_SEED)).cuda()
    cal_syn = torch.empty((ncal, 4, numw), dtype=torch.float64, device="cuda")
    cal_mo = torch.empty_like(cal_m)
    ctx.forward_device(cal_m.data_ptr(), ncal, cal_syn.data_ptr(), cal_mo.data_ptr(), 0, stream=stream,
                       hydrostatic=True)
    cal_gen = torch.Generator(device="cuda")
    cal_gen.manual_seed(CALIB_SEED)
    cal_obs = cal_syn.reshape(ncal, nf) + 1e-3 * torch.randn((ncal, nf), dtype=torch.float64, device="cuda",
                                                             generator=cal_gen)
    ntiles = npix // a.tile
    bufs = {"out": torch.empty((a.tile, 13, a.nz), dtype=torch.float32, device="cuda"),
            "chi": torch.empty(a.tile, dtype=torch.float64, device="cuda"),
            "it": torch.empty(a.tile, dtype=torch.int32, device="cuda"),
            "st": torch.empty(a.tile, dtype=torch.int32, device="cuda")}
    ctx.invert_device(ncal, cal_obs.data_ptr(), base.data_ptr(), bufs["out"].data_ptr(), bufs["chi"].data_ptr(),
                      bufs["it"].data_ptr(), bufs["st"].data_ptr(), hydrostatic=True, opts=opts, stream=stream)
    cal_chi = bufs["chi"][:ncal].clone()
    quants = {"nn": a.accept_quantile, "nn_q10": 0.1, "nn_q30": 0.3}
    levels = {arm: float(torch.quantile(cal_chi, q)) for arm, q in quants.items()}
    accept = {arm: torch.full((a.tile,), t_, dtype=torch.float64, device="cuda") for arm, t_ in levels.items()}
    calib = {"pixels": ncal, "seed": CALIB_SEED, "quantile": a.accept_quantile, "T": levels["nn"],
             "median_chi2": float(torch.median(cal_chi)), "seconds": time.perf_counter() - t0,
             "levels": {arm: {"quantile": quants[arm], "T": levels[arm]} for arm in quants}}
    del cal_m, cal_syn, cal_mo, cal_obs

    results = {"nn": {}, "plain": {}, "free": {}, "tau": {}, "nn_q10": {}, "nn_q30": {}}
    # the reference's own non-learned guess: SET_TAU's T, B and v_z assists
    # on the default model over the tile as a 512 x 256 field
    tau_init = torch.empty_like(base)
    tau_ny = a.field if a.tile == npix else 256
    tau_nx = a.tile // tau_ny
    # the deployable rule: the warm-start model is evaluated once; at or
    # below T it is the result, above T the pixel restarts at once from the
    # default model (fallback_steps -1) and runs plain LM without the goal
    # (fallback_free)
    opts_nn = fz.LMOpts(maxsteps=5, maxit=40, dchi2=1e-3, isigma=1e-3, slots=opts.slots, fallback=1.0,
                        fallback_model=base1.data_ptr(), fallback_steps=-1, fallback_free=True)
    # one output model buffer per (arm, tile), allocated before any timing:
    # the inverted models are compared with the true atmospheres afterwards
    outs = {(arm, k): torch.empty((a.tile, 13, a.nz), dtype=torch.float32, device="cuda")
            for arm in ("plain", "nn", "free", "tau") for k in range(ntiles)}
    outs_tmp = torch.empty((a.tile, 13, a.nz), dtype=torch.float32, device="cuda")

    def step(i, arm):
        k = i % ntiles
        o = obs[k * a.tile:(k + 1) * a.tile]
        if arm == "plain":
            init = base
        elif arm == "tau":
            init = tau_init
            init.copy_(base)
            ctx.set_tau_device(tau_nx, tau_ny, o.data_ptr(), init.data_ptr(), ("temp", "bvec", "vlos"), stream=stream)
        else:
            # network + node expansion in the library (fz_warm_start_device)
            init = nn_init
            warm.models_device(ctx, a.tile, o.data_ptr(), base1.data_ptr(), init.data_ptr(), stream=stream)
        rule = arm in accept
        out_m = outs.get((arm, k), outs_tmp)
        ctx.invert_device(a.tile, o.data_ptr(), init.data_ptr(), out_m.data_ptr(), bufs["chi"].data_ptr(),
                          bufs["it"].data_ptr(), bufs["st"].data_ptr(), hydrostatic=True,
                          opts=opts_nn if rule else opts, stream=stream,
                          target_ptr=accept[arm].data_ptr() if rule else 0)
        results[arm][k] = (bufs["chi"].cpu().numpy().copy(), bufs["it"].cpu().numpy().copy(),
                           int(bufs["st"].max().item()))

    def timed(arm, steps, warmup, tag, profile=False):
        """Warm-up steps, then the timed steps (no per-kernel events: they cost
        host time between launches and keep the iteration out of its CUDA
        graph); with profile, the timed steps once more with the library's
        per-kernel CUDA events on its launching stream, for the kernel times,
        launch counts and columns per launch."""
        for i in range(warmup):
            step(i, arm)
        torch.cuda.synchronize()
        sampler = ClockSampler(local, tag)
        sampler.start()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed_" + tag)   # a profiler can select the timed launches
        e0.record()
        for i in range(a.warmup, a.warmup + steps):
            step(i, arm)
        e1.record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        barrier()
        clocks = sampler.stop()
        prof = None
        if profile:
            ctx.profile(True)
            ctx.profile_read()
            torch.cuda.nvtx.range_push("profiled_" + tag)   # kernels launched one by one, between events
            for i in range(a.warmup, a.warmup + steps):
                step(i, arm)
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
            ctx.profile(False)
            prof = ctx.profile_read(items=True)
        return maxms(e0.elapsed_time(e1) / steps), clocks, prof

    # plain LM from the default guess: the yardstick (the same field; one
    # warm-up step, the graphs and kernels being those of the calibration)
    steps_pl = max(1, min(a.plain_steps, a.steps))
    ms_pl, clocks_pl, _ = timed("plain", steps_pl, 1, "plain")
    plain_value = world * a.tile / (ms_pl * 1e-3)
    # headline: the deployable NN-warm rule at T
    ms_nn, clocks, prof = timed("nn", a.steps, a.warmup, "nn", profile=True)
    value = world * a.tile / (ms_nn * 1e-3)
    sub = max(1, min(a.sub_steps, a.steps))
    ms_sub = {}
    for arm in ("nn_q10", "nn_q30", "free", "tau"):
        ms_sub[arm], _, _ = timed(arm, sub, 0, arm)

    def versus_plain(arm):
        """chi2 and iterations of an arm against plain LM on the same tiles."""
        ks = sorted(set(results[arm]) & set(results["plain"]))
        c = np.concatenate([results[arm][k][0] for k in ks])
        it = np.concatenate([results[arm][k][1] for k in ks])
        cp = np.concatenate([results["plain"][k][0] for k in ks])
        return {"median_chi2": float(np.median(c)), "median_chi2_plain": float(np.median(cp)),
                "mean_iterations": float(it.mean()),
                "frac_pixels_at_or_below_plain_chi2": float(np.mean(c <= cp)),
                "frac_pixels_chi2_above_1.1x_plain": float(np.mean(c > 1.1 * cp)),
                "frac_pixels_chi2_above_2x_plain": float(np.mean(c > 2.0 * cp)),
                "pixels_compared": int(c.size)}

    def sub_arm(arm, definition):
        v = world * a.tile / (ms_sub[arm] * 1e-3)
        return dict(versus_plain(arm), value=v, unit=UNIT, ms_per_step=ms_sub[arm], steps=sub,
                    speedup_vs_plain=v / plain_value, definition=definition)

    common = sorted(set(results["plain"]) & set(results["nn"]) & set(results["free"]) & set(results["tau"]))
    status_bad = max(results[arm][k][2] for arm in results for k in results[arm])
    it_pl = np.concatenate([results["plain"][k][1] for k in sorted(results["plain"])])
    chi_pl = np.concatenate([results["plain"][k][0] for k in sorted(results["plain"])])
    nn_cmp = versus_plain("nn")
    nn_restart = float(np.mean(np.concatenate([results["nn"][k][1] for k in sorted(results["nn"])]) > 1))

    # ------------------------------------------------------ parameter errors
    # errors of the inverted atmospheres against the true ones at the heights
    # where the lines form (log tau5 of the true atmosphere in [-3, 0]);
    # B_perp = |(Bx, By)| (the 180-degree azimuth ambiguity leaves Q, U
    # unchanged under (Bx, By) -> -(Bx, By))
    def height_errors(est, tru):
        tau = tru[:, 11]
        msk = (tau >= -3.0) & (tau <= 0.0)
        e = {}
        for name, d in (("T_K", est[:, 0] - tru[:, 0]), ("Bz_G", est[:, 7] - tru[:, 7]),
                        ("vz_km_s", (est[:, 10] - tru[:, 10]) * 1e-5),
                        ("Bperp_G", torch.hypot(est[:, 5], est[:, 6]) - torch.hypot(tru[:, 5], tru[:, 6]))):
            v = d[msk].double()
            e[name] = {"rms": float(torch.sqrt(torch.mean(v * v))), "median_abs": float(torch.median(v.abs()))}
        return e

    def tiles(src):
        return torch.cat([src(k) for k in common])

    def prior_models(k):
        m_ = torch.empty_like(base)
        warm.models_device(ctx, a.tile, obs[k * a.tile:(k + 1) * a.tile].data_ptr(), base1.data_ptr(), m_.data_ptr(),
                           stream=stream)
        torch.cuda.synchronize()
        return m_

    tru_c = tiles(lambda k: true_models[k * a.tile:(k + 1) * a.tile])
    errors = {arm: height_errors(tiles(lambda k: outs[(arm, k)]), tru_c)
              for arm in ("plain", "nn", "free", "tau")}
    errors["nn_prior"] = height_errors(
        tiles(lambda k: prior_models(k)), tru_c)
    errors["default_guess"] = height_errors(base[:1].expand(tru_c.shape[0], -1, -1), tru_c)
    errors["heights_compared_per_pixel"] = float(((tru_c[:, 11] >= -3.0) & (tru_c[:, 11] <= 0.0)).sum()
                                                 / tru_c.shape[0])

    # ------------------------------------------------------------ errors mode
    # GET_ERROR_1D for the headline arm's inverted models of one tile: the
    # node Jacobian of each model, chi2 and sigma = sqrt(chi2/NFREQ / H_ii)
    # mapped to heights (fz_errors_device)
    k0 = common[0]
    e_m = torch.empty((a.tile, 13, a.nz), dtype=torch.float32, device="cuda")
    e_c = torch.empty(a.tile, dtype=torch.float64, device="cuda")
    e_s = torch.empty(a.tile, dtype=torch.int32, device="cuda")

    def err_call():
        ctx.errors_device(a.tile, obs[k0 * a.tile:(k0 + 1) * a.tile].data_ptr(), outs[("nn", k0)].data_ptr(),
                          e_m.data_ptr(), e_c.data_ptr(), e_s.data_ptr(), hydrostatic=True, opts=opts,
                          stream=stream)

    # the warm-up call in an NVTX range: a profiler can pick its launches,
    # whose k_synth_rf lists every column of the chunk
    torch.cuda.nvtx.range_push("errors_mode")
    err_call()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record()
    for _ in range(2):
        err_call()
    ee1.record()
    torch.cuda.synchronize()
    ms_err = maxms(ee0.elapsed_time(ee1) / 2)
    tru0 = true_models[k0 * a.tile:(k0 + 1) * a.tile]
    msk0 = (tru0[:, 11] >= -3.0) & (tru0[:, 11] <= 0.0)
    errors_mode = {"value": world * a.tile / (ms_err * 1e-3), "unit": "pixels/s", "ms_per_call": ms_err,
                   "workload": "%d inverted pixels (headline arm), NP = 13, %d heights, NFREQ %d: synthesis, "
                               "node Jacobian, chi2, sigma per node, height errors" % (a.tile, a.nz, nf),
                   "median_sigma_T_K": float(torch.median(e_m[:, 0][msk0])),
                   "median_sigma_vz_km_s": float(torch.median(e_m[:, 10][msk0])) * 1e-5,
                   "status_errors": int(e_s.max().item())}
    del outs, e_m, e_c, e_s

    # ------------------------------------------------------------- end to end
    # the headline arm through fz_invert_warm from pinned host memory:
    # observations, the network's standardisation, the default model, T per
    # pixel and the fallback model in; models, chi2, iterations and status
    # out (the network and the LM run on the device between the copies)
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    h_obs = pin((a.tile, 4, numw), torch.float64)
    h_obs[:] = obs[:a.tile].reshape(a.tile, 4, numw).cpu().numpy()
    h_out = (pin((a.tile, 13, a.nz), torch.float32), pin((a.tile,), torch.float64), pin((a.tile,), torch.int32),
             pin((a.tile,), torch.int32))
    e2e_steps = max(1, min(a.steps, 2))
    h_target = pin((a.tile,), torch.float64)
    h_target[:] = levels["nn"]
    h_base = pin((13, a.nz), torch.float32)
    h_base[:] = base1.cpu().numpy()
    opts_e2e = fz.LMOpts(maxsteps=5, maxit=40, dchi2=1e-3, isigma=1e-3, slots=opts.slots, fallback=1.0,
                         fallback_model=h_base.ctypes.data, fallback_steps=-1,
                         fallback_free=True)   # a host pointer for the host-buffer call
    warm._hnorm = warm.norm()

    def e2e_step():
        ctx.invert_warm(h_obs, warm, base=h_base, hydrostatic=True, opts=opts_e2e, target=h_target, out=h_out)

    e2e_step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    ms_e2e = maxms((time.perf_counter() - t0) * 1e3 / e2e_steps)
    nm_ = 13 * a.nz
    e2e = {"value": world * a.tile / (ms_e2e * 1e-3), "unit": UNIT, "steps": e2e_steps,
           "h2d_bytes_per_step": a.tile * nf * 8 + a.tile * 8 + warm._hnorm.nbytes + 2 * nm_ * 4,
           "d2h_bytes_per_step": a.tile * nm_ * 4 + a.tile * (8 + 4 + 4),
           "note": "the headline arm through fz_invert_warm (one C-ABI call per step): host observations, "
                   "standardisation, default model, T per pixel and fallback model in; models, chi2, iterations "
                   "and status out; pinned host buffers; wall clock around the calls"}

    # --------------------------------------------------------- synthesis rate
    ns = a.synth_cols
    m = torch.from_numpy(fz.atmos.make_columns(ns, a.nz, seed=2 + rank)).cuda()
    so = torch.empty((ns, 4, numw), dtype=torch.float64, device="cuda")
    mo = torch.empty_like(m)
    for _ in range(3):
        ctx.forward_device(m.data_ptr(), ns, so.data_ptr(), mo.data_ptr(), 0, stream=stream, hydrostatic=True)
    torch.cuda.synchronize()
    ctx.profile(True)
    ctx.profile_read()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        ctx.forward_device(m.data_ptr(), ns, so.data_ptr(), mo.data_ptr(), 0, stream=stream, hydrostatic=True)
    e1.record()
    torch.cuda.synchronize()
    ctx.profile(False)
    sprof_items = ctx.profile_read(items=True)
    sprof = {k: v[:2] for k, v in sprof_items.items()}
    ms_syn = maxms(e0.elapsed_time(e1) / 5)
    synthesis = {"value": world * ns * numw / (ms_syn * 1e-3), "unit": "columns*lambda/s",
                 "workload": "%d columns x %d heights x %d lambda, hydrostatic" % (ns, a.nz, numw),
                 "ms_per_call": ms_syn, "kernel_ms": {k: v[0] / max(v[1], 1) for k, v in sprof.items() if v[1]}}
    # ------------------------------------ synthesis with a line spread function
    # the same columns with the reference's Gaussian LSF (sigma 30 mA) in both
    # regions: k_lsf convolves each Stokes row region by region in FP64
    # (2 n^2 FLOP per region row, n = NUMWAVE)
    for r in range(len(ctx.regions)):
        ctx.lsf_gaussian(r, 30.0, 0.0)
    ctx.forward_device(m.data_ptr(), ns, so.data_ptr(), mo.data_ptr(), 0, stream=stream, hydrostatic=True)
    torch.cuda.synchronize()
    ctx.profile(True)
    ctx.profile_read()
    e0.record()
    for _ in range(5):
        ctx.forward_device(m.data_ptr(), ns, so.data_ptr(), mo.data_ptr(), 0, stream=stream, hydrostatic=True)
    e1.record()
    torch.cuda.synchronize()
    ctx.profile(False)
    lprof = ctx.profile_read()
    ctx.lsf_clear()
    ms_lsf = maxms(e0.elapsed_time(e1) / 5)
    k_lsf_ms = lprof["k_lsf"][0] / max(lprof["k_lsf"][1], 1)
    lsf_flop = ns * 4 * sum(2.0 * int(n) ** 2 for n in ctx.regions["numwave"])
    synthesis_lsf = {"value": world * ns * numw / (ms_lsf * 1e-3), "unit": "columns*lambda/s",
                     "workload": synthesis["workload"] + ", Gaussian LSF sigma 30 mA in every region",
                     "ms_per_call": ms_lsf, "k_lsf_ms": k_lsf_ms,
                     "k_lsf_fp64_gflops": lsf_flop / (k_lsf_ms * 1e-3) / 1e9,
                     "k_lsf_gbs": ns * nf * 8 * 2 / (k_lsf_ms * 1e-3) / 1e9}
    # ------------------------------- response functions at every height (C2)
    # 256x256 columns (the synthesis sub-metric's) through fz_forward_rf_full
    # in batches of rf_chunk columns; each batch's output (rf_chunk x 6 x NZ x
    # NFREQ float32, 11.3 GB at 4096) is overwritten by the next
    rc_ = min(a.rf_chunk, ns)
    rfo = torch.empty((rc_, 6, a.nz, nf), dtype=torch.float32, device="cuda")
    sor = torch.empty((rc_, 4, numw), dtype=torch.float64, device="cuda")
    mor = torch.empty((rc_, 13, a.nz), dtype=torch.float32, device="cuda")
    nb_rf = ns // rc_

    def rf_batch(i):
        ctx.forward_rf_full_device(m[i * rc_:(i + 1) * rc_].data_ptr(), rc_, sor.data_ptr(), rfo.data_ptr(),
                                   mor.data_ptr(), 0, stream=stream, hydrostatic=True)

    rf_batch(0)
    torch.cuda.synchronize()
    ctx.profile(True)
    ctx.profile_read()
    e0.record()
    for i in range(nb_rf):
        rf_batch(i)
    e1.record()
    torch.cuda.synchronize()
    ctx.profile(False)
    rprof = ctx.profile_read()
    ms_rf = maxms(e0.elapsed_time(e1))
    rf_full = {"value": world * nb_rf * rc_ * numw / (ms_rf * 1e-3), "unit": "columns*lambda/s",
               "workload": "%d columns x %d heights x %d lambda, hydrostatic, RFs to T, Pg, Bx, By, Bz, v_z at "
                           "every height (fz_forward_rf_full, %d columns per call)" % (nb_rf * rc_, a.nz, numw, rc_),
               "ms_total": ms_rf, "rf_bytes_per_column": 6 * a.nz * nf * 4,
               "kernel_ms": {k: v[0] / max(v[1], 1) for k, v in rprof.items() if v[1]},
               "error_vs_oracle": "tests/test_gpu_rf.py: every (column, parameter, height) within 2e-3 of the "
                                  "parameter's largest response; Stokes I 1e-5 relative, Q/U/V 1e-6 I_c"}
    del rfo, sor, mor
    torch.cuda.empty_cache()

    # --------------------------------------------------------------- v3 files
    # the reference's file formats around the path: the GPU layout changes of
    # one tile (profile file payload -> OBS3D, synthesis -> profile payload,
    # model-file cubes <-> MODEL) and of 1,024 columns of full-height RFs ->
    # the RF file payload, timed with CUDA events (5 calls after one warm-up;
    # bytes = what each kernel must read + write), and the host record I/O of
    # a 16,384-pixel slice on a RAM-backed directory (wall clock)
    from firtez_dz_b200 import v3io
    nyv = 256
    nxv = a.tile // nyv
    tst = torch.zeros((nxv, nyv, numw, 4), dtype=torch.float32, device="cuda")
    tob = torch.empty((a.tile, 4, numw), dtype=torch.float64, device="cuda")
    tcu = torch.zeros((13, nxv, nyv, a.nz), dtype=torch.float32, device="cuda")
    tmo = torch.empty((a.tile, 13, a.nz), dtype=torch.float32, device="cuda")
    ncr = 1024
    trf = torch.zeros((ncr, 6, a.nz, nf), dtype=torch.float32, device="cuda")
    tro = torch.empty((ncr, 1, a.nz, numw, 4, 6), dtype=torch.float32, device="cuda")
    xs, ys = np.arange(nxv) * 16.0, np.arange(nyv) * 16.0
    layout = {
        "obs_from_profile_file": (lambda: v3io.obs_from_stokes_device(tst, out=tob, stream=stream),
                                  a.tile * numw * 4 * (4 + 8)),
        "syn_to_profile_file": (lambda: v3io.stokes_from_syn_device(tob, nxv, nyv, out=tst, stream=stream),
                                a.tile * numw * 4 * (8 + 4)),
        "model_from_model_file": (lambda: v3io.model_from_cubes_device(tcu, out=tmo, stream=stream),
                                  a.tile * 13 * a.nz * 4 * 2),
        "model_to_model_file": (lambda: v3io.cubes_from_model_device(tmo, nxv, nyv, xs, ys, out=tcu, stream=stream),
                                a.tile * 13 * a.nz * 4 * 2),
        "rf_full_to_rf_file": (lambda: v3io.rf_file_layout_device(trf, ncr, 1, out=tro, stream=stream),
                               ncr * 6 * a.nz * nf * 4 * 2),
    }
    hbm_pk, hbm_how = peaks()
    v3_kernels = {}
    for name, (fn, nbytes) in layout.items():
        fn()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(5):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        ms_k = maxms(ev0.elapsed_time(ev1) / 5)
        v3_kernels[name] = {"ms": ms_k, "bytes": nbytes, "gbs": nbytes / (ms_k * 1e-3) / 1e9,
                            "frac_hbm": nbytes / (ms_k * 1e-3) / 1e9 / hbm_pk}
    v3_kernels["model_to_model_file"]["note"] = ("includes the copy of the x, y vectors to the device and the "
                                                 "call's stream synchronisation")
    del tst, tob, tcu, tmo, trf, tro
    torch.cuda.empty_cache()
    import tempfile
    nsl = 16384
    base_dir = "/dev/shm" if os.path.isdir("/dev/shm") else None
    rng_v3 = np.random.default_rng(7)
    h_st = rng_v3.standard_normal((nsl // nyv, nyv, numw, 4)).astype(np.float32)
    h_cu = rng_v3.standard_normal((13, nsl // nyv, nyv, a.nz)).astype(np.float32)
    host_io = {}
    with tempfile.TemporaryDirectory(dir=base_dir) as td:
        for kind, wr, rd, nbytes in (
                ("profile", lambda f: v3io.write_profile(f, np.ones(numw), np.arange(numw, dtype=np.float64), h_st),
                 v3io.read_profile, h_st.nbytes),
                ("model", lambda f: v3io.write_model(f, h_cu), v3io.read_model, h_cu.nbytes)):
            fn_ = os.path.join(td, kind + ".bin")
            t0 = time.perf_counter()
            wr(fn_)
            t1 = time.perf_counter()
            rd(fn_)
            t2 = time.perf_counter()
            host_io[kind] = {"bytes": nbytes, "write_mb_s": nbytes / (t1 - t0) / 1e6,
                             "read_mb_s": nbytes / (t2 - t1) / 1e6}
    v3_files = {"layout_kernels": v3_kernels, "peak_gbs": hbm_pk, "peak_source": hbm_how,
                "workload": "one %d-pixel tile (%d x %d), NZ %d, NUMW %d; RFs: %d columns" % (a.tile, nxv, nyv,
                                                                                              a.nz, numw, ncr),
                "host_record_io": dict(host_io, slice_pixels=nsl, directory=base_dir or "tempfile default")}

    # ------------------------------------------------ four-line workload (C5)
    del obs, true_models, outs_tmp
    torch.cuda.empty_cache()
    c5 = c5_sub_metric(a, fz, rank, world, stream, maxms) if a.c5_tiles > 0 else None

    if rank != 0:
        ranks.close()
        return

    # -------------------------------------------------------------- roofline
    # each kernel of the FLOP table against its pipe (FP32 or FP64 FLOP per
    # column counted by ncu x mean columns per launch / mean launch time,
    # over the peak of an FMA-chain kernel measured here); HBM as the side
    # figure: algorithmic bytes per column x columns / launch time
    hbm, how = peaks()
    fp32 = fz.measure_fp32_peak(local)
    fp64 = fz.measure_fp64_peak(local)
    pipe_peak = {"fp32": fp32, "fp64": fp64}
    flops_tab, traffic_tab = {}, {}
    for fn_, dst in (("flops.json", flops_tab), ("traffic.json", traffic_tab)):
        pth = os.path.join(ROOT, "profiles", fn_)
        if os.path.exists(pth):
            d_ = json.load(open(pth))
            dst.update(d_.get("kernels", d_))

    def launch_means(pr):
        return {k: (v[0] / max(v[1], 1), v[1], v[2] / max(v[1], 1)) for k, v in pr.items() if v[1]}

    def pipe_lines(pr):
        out_ = {}
        for k, (kms_, n_, cols_) in launch_means(pr).items():
            e_ = flops_tab.get(k)
            if not isinstance(e_, dict):
                continue
            ach = e_["flop_per_column"] * cols_ / (kms_ * 1e-3) / 1e12
            out_[k] = {"pipe": e_["pipe"], "achieved_tflops": ach, "peak_tflops": pipe_peak[e_["pipe"]],
                       "frac": ach / pipe_peak[e_["pipe"]], "mean_launch_ms": kms_, "launches": n_,
                       "mean_columns_per_launch": cols_}
        return out_

    per_launch = launch_means(prof)
    kname = max(prof, key=lambda k: prof[k][0])
    kms, _, cols = per_launch[kname]            # mean launch time, mean columns per launch
    np_ = 13
    if kname == "k_synth_rf":
        alg_col = a.nz * 6 * 4 + nf * 8 + np_ * nf * 4      # model in, RSYN1D + EQVDSYN out
    elif kname in ("k_opac_rf", "k_chemder"):
        alg_col = a.nz * 7 * 4                               # T, Pg, rho, Bx, By, Bz, vz in
    elif kname == "k_chain":
        alg_col = a.nz * (3 * 4 + 4 * 4 + 16)                # T, Pg, z in; Pg, rho, Pe, mu, (nH, ne) out
    elif kname == "k_synth":
        alg_col = nf * 8 + a.nz * 4                          # RSYN1D and log tau5 out
    else:
        alg_col = a.nz * 6 * 4
    hbm_ach = alg_col * cols / (kms * 1e-3) / 1e9
    traffic = traffic_tab.get(kname) * cols if isinstance(traffic_tab.get(kname), (int, float)) else None
    pipes = pipe_lines(prof)
    if kname in pipes:
        pl_ = pipes[kname]
        roofline = {"bound": pl_["pipe"], "kernel": kname, "achieved": pl_["achieved_tflops"],
                    "peak": pl_["peak_tflops"], "unit": "TFLOP/s", "frac": pl_["frac"], "traffic": traffic,
                    "peak_source": "measured in this run: FMA-chain kernel (fz_measure_%s_peak), of measured"
                                   % pl_["pipe"],
                    "flop_per_column": flops_tab[kname]["flop_per_column"],
                    "flop_source": "ncu thread-level ffma/fadd/fmul (dfma/dadd/dmul) counts, an FMA as 2, on "
                                   "2048 columns of this workload (profiles/flops.json)",
                    "mean_launch_ms": kms, "mean_columns_per_launch": cols,
                    "hbm_side": {"achieved_gbs": hbm_ach, "peak_gbs": hbm, "frac": hbm_ach / hbm,
                                 "algorithmic_bytes_per_launch": alg_col * cols,
                                 "peak_source": how + " (MEASURED_PEAKS.json hbm_gbs)" if how == "measured" else how}}
    else:
        roofline = {"bound": "hbm", "kernel": kname, "achieved": hbm_ach, "peak": hbm, "unit": "GB/s",
                    "frac": hbm_ach / hbm, "traffic": traffic,
                    "peak_source": how + " (MEASURED_PEAKS.json hbm_gbs)" if how == "measured" else how,
                    "algorithmic_bytes_per_launch": alg_col * cols, "mean_launch_ms": kms,
                    "mean_columns_per_launch": cols}
    synthesis["pipe_rooflines"] = pipe_lines(sprof_items)
    nchunk = -(-a.tile // 16384)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": ms_nn, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
           "data": "synthetic (seeded atmospheres, firtez-dz_b200/atmos.py; observations = GPU synthesis + "
                   "1e-3 noise)",
           "config": dict(config, autotuned=tuned if tuned else "off (--no-tune): slots %d" % a.slots),
           "definition": "pixels/s of the deployable NN-warm rule: the warm-start model of every pixel is "
                         "evaluated once and kept where its chi2 <= T (T = the %.2f quantile of plain-LM chi2 on "
                         "a separate %d-pixel calibration set inverted before the timed region); every other "
                         "pixel restarts at once from the default guess in the same slot pool and runs plain LM "
                         "(the reference's stop rules)" % (a.accept_quantile, ncal),
           "calibration": calib,
           "plain": {"value": plain_value, "unit": UNIT, "ms_per_step": ms_pl,
                     "median_chi2": float(np.median(chi_pl)), "mean_iterations": float(it_pl.mean()),
                     "clocks": clocks_pl},
           "nn_warm": dict(nn_cmp, value=value, speedup_vs_plain=value / plain_value,
                           frac_pixels_restarted=nn_restart, status_errors=status_bad, mlp=mlp_info,
                           note="mean_iterations counts the evaluation of the warm-start model as one; a "
                                "restarted pixel adds its plain-LM iterations"),
           "nn_warm_q10": sub_arm("nn_q10", "the headline rule with T at the 0.10 quantile"),
           "nn_warm_q30": sub_arm("nn_q30", "the headline rule with T at the 0.30 quantile"),
           "nn_warm_free": sub_arm("free", "NN-warm LM with the plain stop rules only"),
           "set_tau_plain": sub_arm("tau", "LM with the plain stop rules from the default model after "
                                           "SET_TAU's T, B and v_z assists over the tile (the reference's "
                                           "non-learned initial guess)"),
           "parameter_errors": dict(errors, definition="errors of T, Bz, v_z and |B_perp| of the inverted "
                                           "atmospheres against the true ones at the heights where the true "
                                           "log tau5 is in [-3, 0], over the compared pixels"),
           "synthesis": synthesis,
           "rf_full": rf_full,
           "synthesis_lsf": synthesis_lsf,
           "errors_mode": errors_mode,
           "v3_files": v3_files,
           "four_lines_c5": c5,
           "roofline": roofline,
           "pipe_rooflines": pipes,
           "kernel_ms": {k: v[0] for k, v in per_launch.items()},
           "kernel_share": {k: prof[k][0] / sum(v[0] for v in prof.values()) for k in per_launch},
           "kernel_timing": "per-kernel CUDA events of the library on its launching stream, over a repetition "
                            "of the timed headline steps (the timed pass itself runs without them)",
           "kernel_launches": {k: v[1] for k, v in per_launch.items()},
           "kernel_columns_per_launch": {k: v[2] for k, v in per_launch.items()},
           "e2e": e2e,
           # kernels counted by the context plus, per step, the warm start:
           # per 16384-pixel chunk one conversion + 4 GEMMs, then CONTRACT of
           # the base model and the node expansion
           "gpu_launches": int(sum(v[1] for v in prof.values()) + (5 * nchunk + 2) * a.steps),
           "clocks": clocks}
    if world == 1:
        # the oracle on the host cores, with its own line parse (the same rows)
        olines, oreg = cpu_workload()
        npx = a.cpu_pixels if a.cpu_pixels > 0 else 4 * os.cpu_count()
        v, el, c = cpu_lm_sample(olines, oreg, he, a.nz, npx, seed=1000)
        sv, sel = cpu_synth_sample(olines, oreg, he, a.nz, 256, seed=2)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                               "sample": "%d pixels (4 x cores), LM from the default guess, in %.1f s (FP64 C++ "
                                         "restatement of the reference's forward/RF routines, OpenMP over pixels, "
                                         "+ numpy/LAPACK LM); median chi2 %.3g" % (npx, el, c),
                               "synthesis": {"value": sv, "unit": "columns*lambda/s", "seconds": sel,
                                             "workload": "256 columns x %d heights x %d lambda, hydrostatic, "
                                                         "FP64" % (a.nz, numw),
                                             "gpu_over_cpu": synthesis["value"] / sv}}
    print(json.dumps(out))
    sys.stdout.flush()
    ranks.close()


if __name__ == "__main__":
    main()
