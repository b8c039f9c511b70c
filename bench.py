#!/usr/bin/env python3
"""Benchmark of the GPU Stokes synthesis (FORWARD3D/FORWARD1D batched on one B200).

Workload: 256 x 256 columns x 128 heights, Fe I 6301.5 + 6302.5 x 112 points
each (NUMW = 224), hydrostatic equilibrium integrated on the GPU in FP64
(RK4 from the top), chemical equilibrium FP64, opacities / Voigt / formal
solution FP32.  Seeded synthetic atmospheres (firtez-dz_b200/atmos.py).

One step = one synthesis of all columns.  ``value`` = columns x wavelengths
per second with inputs resident in HBM; ``e2e`` = the same through the
host-buffer C-ABI call (fz_forward) with the model copied from pinned host
memory and RSYN1D copied back every step.  Multi-GPU: every rank synthesises
its own 256 x 256 tile (weak scaling, no collective on the data path).

``--impl reference`` times the CPU restatement of the reference (the Fortran
reference cannot be built on this image: no gfortran/MPI/LAPACK) on all host
cores, on bounded samples of the same workload.
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
UNIT = "columns*lambda/s"


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

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", "clocks_rank%d.csv" % index)

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


def cpu_sample(lines, reg, gain, model, hydrostatic, budget_s):
    """Oracle on consecutive 64-column batches until budget_s; cols*lambda/s."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import orc
    numw = int(reg["numwave"].sum())
    done, t0, i = 0, time.perf_counter(), 0
    while True:
        batch = model[(i * 64) % len(model):(i * 64) % len(model) + 64]
        orc.forward(lines, reg, gain, batch, hydrostatic=hydrostatic, nthreads=0)
        done += len(batch)
        i += 1
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    return done * numw / el, done, el


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ncol", type=int, default=256 * 256)
    ap.add_argument("--nz", type=int, default=128)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-he", action="store_true")
    a = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    he = not a.no_he
    fz = load_package()
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    numw = int(reg["numwave"].sum())
    config = {"workload": "synthesis %dx%d columns x %d heights, Fe I 6301.5+6302.5 x 112 lambda, "
                          "hydrostatic FP64 + chemistry FP64, RTE FP32" % (int(np.sqrt(a.ncol)), int(np.sqrt(a.ncol)), a.nz),
              "columns_per_gpu": a.ncol, "nz": a.nz, "numw": numw, "hydrostatic": he,
              "l2": "inputs larger than L2 (model %.0f MB per GPU)" % (a.ncol * 13 * a.nz * 4 / 1e6),
              "parallelism": "columns sharded per GPU" if world > 1 else "single GPU"}

    if a.impl == "reference":
        if rank != 0:
            return
        model = fz.atmos.make_columns(min(a.ncol, 4096), a.nz, seed=2)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import orc
        gain, _ = orc.gain(lines, reg)
        vals = []
        for _ in range(a.warmup):
            cpu_sample(lines, reg, gain, model, he, 0.5)
        per = max(a.cpu_seconds / max(a.steps, 1), 1.0)
        tot_cols = tot_t = 0.0
        for _ in range(a.steps):
            v, n, el = cpu_sample(lines, reg, gain, model, he, per)
            vals.append(v)
            tot_cols += n
            tot_t += el
        value = float(np.mean(vals))
        cores = os.cpu_count()
        out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
               "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot_t / a.steps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic", "config": config,
               "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": "%d columns of the workload per step, OpenMP over columns "
                                          "(FP64 C++ restatement; the Fortran reference needs gfortran/MPI/LAPACK, "
                                          "absent on this image)" % int(tot_cols / a.steps)},
               "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    model = fz.atmos.make_columns(a.ncol, a.nz, seed=2 + rank)
    ctx = fz.Synthesis(lines, reg, nz=a.nz, device=local)
    d_model = torch.from_numpy(model).cuda()
    d_out = torch.empty_like(d_model)
    d_syn = torch.empty((a.ncol, 4, numw), dtype=torch.float64, device="cuda")
    d_st = torch.zeros(a.ncol, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        ctx.forward_device(d_model.data_ptr(), a.ncol, d_syn.data_ptr(), d_out.data_ptr(), d_st.data_ptr(),
                           stream=stream, hydrostatic=he)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    assert int(d_st.max().item()) == 0, "column status errors"
    sampler = ClockSampler(local)
    sampler.start()
    ctx.profile(True)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    ctx.profile(False)
    prof = ctx.profile_read()
    ms = e0.elapsed_time(e1) / a.steps
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * a.ncol * numw / (ms * 1e-3)

    # end to end through the host-buffer C-ABI call, pinned host memory
    h_model = torch.from_numpy(model).pin_memory()
    h_syn = torch.empty((a.ncol, 4, numw), dtype=torch.float64).pin_memory()
    h_st = torch.empty(a.ncol, dtype=torch.int32).pin_memory()
    L = fz.lib()

    def e2e_step():
        rc = L.fz_forward(ctx._h, a.ncol, h_model.data_ptr(), int(he), h_syn.data_ptr(), None, h_st.data_ptr())
        if rc < 0:
            raise fz.FzError(L.fz_strerror(rc).decode())

    for _ in range(max(1, a.warmup)):
        e2e_step()
    barrier()
    torch.cuda.synchronize()
    e2 = max(1, a.steps // 2)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(e2):
        e2e_step()
    t1.record()
    torch.cuda.synchronize()
    ms_e2e = t0.elapsed_time(t1) / e2
    if dist is not None:
        t = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = {"value": world * a.ncol * numw / (ms_e2e * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": a.ncol * 13 * a.nz * 4,
           "d2h_bytes_per_step": a.ncol * 4 * numw * 8 + a.ncol * 4}
    assert int(h_st.max()) == 0

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # roofline of the dominant kernel (algorithmic bytes per launch / mean launch time)
    hbm, how = peaks()
    kname = max(prof, key=lambda k: prof[k][0])
    kms = prof[kname][0] / max(prof[kname][1], 1)
    if kname == "k_chain":
        alg = a.ncol * (2 + 4) * a.nz * 4        # T,Pg in; Pg,rho,Pe,mu out
    elif kname == "k_opac":
        alg = a.ncol * (5 * 4) * a.nz            # T,Bx,By,Bz,vz in (nH, ne and the slab are intermediates)
    else:
        alg = a.ncol * 4 * numw * 8              # RSYN1D out (the slab is an intermediate)
    achieved = alg / (kms * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            per_col = json.load(open(tf)).get(kname)
            traffic = per_col * a.ncol if per_col else None
        except Exception:
            traffic = None
    fp32 = fz.measure_fp32_peak(local)
    flop_synth = a.ncol * a.nz * numw * (145.0 * 8 + 200.0)
    synth_ms = prof["k_synth"][0] / max(prof["k_synth"][1], 1)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
           "data": "synthetic (seeded atmospheres, firtez-dz_b200/atmos.py)", "config": config,
           "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                        "frac": achieved / hbm, "traffic": traffic,
                        "peak_source": how + " (MEASURED_PEAKS.json hbm_gbs)" if how == "measured" else how,
                        "algorithmic_bytes_per_launch": alg, "mean_launch_ms": kms},
           "fp32_roofline": {"kernel": "k_synth", "achieved_tflops": flop_synth / (synth_ms * 1e-3) / 1e12,
                             "peak_tflops": fp32, "frac": flop_synth / (synth_ms * 1e-3) / 1e12 / fp32,
                             "flop_model": "(145*NTOT_mean + 200) per column*height*lambda, NTOT_mean=8",
                             "peak_source": "measured FMA-chain kernel (fz_measure_fp32_peak)"},
           "kernel_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
           "e2e": e2e, "gpu_launches": sum(v[1] for v in prof.values()), "clocks": clocks}
    if world == 1:
        cps, n, el = cpu_sample(lines, reg, ctx.gain, model, he, a.cpu_seconds)
        out["cpu_baseline"] = {"value": cps, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                               "sample": "%d columns of the workload in %.1f s (FP64 C++ restatement of the "
                                         "reference, OpenMP over columns)" % (n, el)}
    print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
