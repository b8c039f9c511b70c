"""The bench's multi-GPU plumbing on CPU: two gloo ranks.

bench.py --gpus N runs one process per GPU, each inverting a field of its
own (weak scaling); the ranks share only a barrier and the maximum over ranks
of each measured time.  Here two processes on the gloo backend check that
the maximum reaches both ranks, that the barrier and the teardown work, that
the ranks' fields are seeded differently, and that the reference arm's
non-zero ranks exit at once without output.
"""
import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("fz_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    bench = _bench()
    r = bench.Ranks(world, backend="gloo", device="cpu", timeout_s=60)
    r.barrier()
    got = r.maxms(10.0 + 5.0 * rank)
    r.barrier()
    r.close()
    with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
        json.dump({"max": got, "seed": bench.field_seed(rank, 0)}, f)


def test_two_gloo_ranks_share_the_max_time(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(os.path.join(tmp_path, "rank%d.json" % r))) for r in range(world)]
    assert all(x["max"] == 15.0 for x in res)
    assert len({x["seed"] for x in res}) == world


def test_single_rank_needs_no_process_group():
    bench = _bench()
    r = bench.Ranks(1)
    r.barrier()
    assert r.maxms(3.5) == 3.5
    r.close()


@pytest.mark.timeout(300)
def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=280)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


@pytest.mark.timeout(300)
def test_reference_arm_loads_nothing_of_the_product():
    """The reference arm times the oracle alone: after a (small) run of it the
    process has mapped oracle/liborc.so and never the product's
    libfzb200.so, and the package module was never imported."""
    code = ("import sys, json, types; sys.path.insert(0, %r); import importlib.util as u; "
            "s = u.spec_from_file_location('fz_bench', %r); b = u.module_from_spec(s); s.loader.exec_module(b); "
            "a = types.SimpleNamespace(cpu_pixels=2, warmup=0, steps=1, nz=32, gpus=1); "
            "b.reference_arm(a, {}, True); maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'orc': 'liborc.so' in maps, 'fz': 'libfzb200' in maps, "
            "'pkg': 'firtez_dz_b200' in sys.modules}))") % (ROOT, os.path.join(ROOT, "bench.py"))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=280)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = p.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["cpu_baseline"]["kind"] == "port"
    got = json.loads(lines[-1])
    assert got == {"orc": True, "fz": False, "pkg": False}


def test_flops_table_from_an_ncu_csv(tmp_path):
    """--flops-from: thread-level opcode counts of an ncu CSV -> FLOP per
    column (an FMA as 2), the pipe with more FLOP, the median launch."""
    bench = _bench()
    hdr = ["ID", "Kernel Name", "Metric Name", "Metric Value"]
    rows = []
    for i, (name, ffma, dfma) in enumerate((("void k_synth_rf<1, 0, 256, 0>(int)", 1000, 4),
                                            ("void k_chain<1, 32>(int)", 2, 500),
                                            ("void k_chain<1, 16>(int)", 2, 700),
                                            ("void k_chain<1, 32>(int)", 2, 600))):
        for op, v in (("ffma", ffma), ("fadd", 10), ("fmul", 20), ("dfma", dfma), ("dadd", 0), ("dmul", 0)):
            rows.append([str(i), name, "smsp__sass_thread_inst_executed_op_%s_pred_on.sum" % op, "{:,}".format(v)])
        rows.append([str(i), name, "gpu__time_duration.sum", "1000"])
    csvf = tmp_path / "f.csv"
    csvf.write_text("==PROF== banner\n" + "\n".join(",".join('"%s"' % c for c in r) for r in [hdr] + rows) + "\n")
    out = tmp_path / "flops.json"
    bench.flops_table(str(csvf), 10, 2, 5, str(out))
    k = json.load(open(out))["kernels"]
    assert k["k_synth_rf"]["pipe"] == "fp32" and k["k_synth_rf"]["flop_per_column"] == (2000 + 30) / 10
    assert k["k_chain"]["pipe"] == "fp64" and k["k_chain"]["launches"] == 3
    assert k["k_chain"]["flop_per_column"] == 1200 / 10          # the median of 1000, 1200, 1400
    assert k["k_synth_rf"]["flop_per_column_height_lambda"] == k["k_synth_rf"]["flop_per_column"] / 10


def test_flops_table_merges_the_small_batch_kernels(tmp_path):
    """A probe of at most 1,024 columns runs the chain on precomputed Saha
    factors: its capture (k_saha + k_chain) adds k_saha and k_chain_pre to
    the table of the full-batch probe, and a later full-batch table keeps
    them."""
    bench = _bench()
    hdr = ["ID", "Kernel Name", "Metric Name", "Metric Value"]

    def capture(path, kernels):
        rows = []
        for i, (name, dfma) in enumerate(kernels):
            for op, v in (("ffma", 1), ("fadd", 0), ("fmul", 0), ("dfma", dfma), ("dadd", 0), ("dmul", 0)):
                rows.append([str(i), name, "smsp__sass_thread_inst_executed_op_%s_pred_on.sum" % op, str(v)])
        path.write_text("\n".join(",".join('"%s"' % c for c in r) for r in [hdr] + rows) + "\n")

    out = tmp_path / "flops.json"
    full, small = tmp_path / "full.csv", tmp_path / "small.csv"
    capture(full, (("void k_chain<1, 16, 0>(int)", 900), ("void k_synth(int)", 0)))
    capture(small, (("void k_saha<1>(int)", 300), ("void k_chain<1, 32, 1>(int)", 500)))
    bench.flops_table(str(full), 10, 2, 5, str(out))
    bench.flops_table(str(small), 10, 2, 5, str(out))
    k = json.load(open(out))["kernels"]
    assert k["k_chain"]["flop_per_column"] == 180 and k["k_saha"]["flop_per_column"] == 60
    assert k["k_chain_pre"]["flop_per_column"] == 100 and "k_synth" in k
    bench.flops_table(str(full), 10, 2, 5, str(out))
    k = json.load(open(out))["kernels"]
    assert k["k_chain"]["flop_per_column"] == 180 and k["k_chain_pre"]["flop_per_column"] == 100
