"""A field split over ranks by x (firtez-dz_b200/parallel.py) on CPU: the
shard rule of SMOOTHING_B (oracle restatement) equals the whole field's
SMOOTHING_B on the interior columns, and FieldShard's halo exchange over two
and three gloo ranks, with the oracle's shard smoothing standing in for the
GPU kernel, reproduces the whole field's SMOOTHING_B exactly."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import lm_oracle as lmo  # noqa: E402

PARAMS = (1, 4, 6, 7)


def _field(nx, ny, nz, seed=0):
    return np.random.default_rng(seed).standard_normal((nx * ny, 13, nz)).astype(np.float32) * 100


def _parallel():
    from conftest import load_package
    load_package()
    from firtez_dz_b200 import parallel
    return parallel


@pytest.mark.parametrize("nx,world", [(7, 2), (5, 3), (4, 2), (9, 4), (12, 1)])
def test_shard_rule_equals_whole_field(nx, world):
    ny, nz = 5, 6
    par = _parallel()
    full = _field(nx, ny, nz)
    want = lmo.smoothing_b(full, nx, ny, PARAMS)
    for x0, x1 in par.split(nx, world):
        a, b = max(0, x0 - 1), min(nx, x1 + 1)          # with the halo columns
        ext = full[a * ny:b * ny]
        got = lmo.smoothing_b_shard(ext, b - a, ny, a, nx, PARAMS)
        np.testing.assert_array_equal(got[(x0 - a) * ny:(x1 - a) * ny], want[x0 * ny:x1 * ny])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, nx, ny, nz, outdir):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    par = _parallel()
    sh = par.FieldShard(nx, ny, rank, world)
    full = _field(nx, ny, nz)
    local = torch.from_numpy(full[sh.x0 * ny:sh.x1 * ny].copy())
    sh.smooth(local, par.host_smoother(lmo.smoothing_b_shard, PARAMS))
    np.save(os.path.join(outdir, "r%d.npy" % rank), local.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("nx,world", [(7, 2), (8, 3)])
def test_field_shard_gloo_equals_whole_field(tmp_path, nx, world):
    import torch.multiprocessing as mp
    ny, nz = 5, 6
    mp.spawn(_rank, args=(world, _free_port(), nx, ny, nz, str(tmp_path)), nprocs=world, join=True)
    got = np.concatenate([np.load(os.path.join(tmp_path, "r%d.npy" % r)) for r in range(world)], 0)
    np.testing.assert_array_equal(got, lmo.smoothing_b(_field(nx, ny, nz), nx, ny, PARAMS))


def _tau_rank(rank, world, port, nx, n, outdir):
    """SET_TAU's field reductions (FieldShard.field_reduce) on gloo ranks:
    the per-column sums of this rank's columns in, the field total out; the
    rank's maxima in, the field maxima out."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    par = _parallel()
    sh = par.FieldShard(nx, 3, rank, world)
    cols = np.random.default_rng(5).standard_normal((nx, n)) * 10 ** np.random.default_rng(6).uniform(-3, 3, (nx, 1))
    fn = sh.field_reduce()
    buf = np.zeros(max(sh.nx * n, 3))
    buf[:sh.nx * n] = cols[sh.x0:sh.x1].ravel()
    assert fn(0, buf, n, sh.nx) == 0
    total = buf[:n].copy()
    mx = np.array([rank + 0.5, 10.0 - rank, 2.0 * rank])
    assert fn(1, mx, 3, 1) == 0
    np.save(os.path.join(outdir, "t%d.npy" % rank), np.concatenate([total, mx]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("nx,world", [(7, 2), (8, 3)])
def test_set_tau_field_reductions_gloo(tmp_path, nx, world):
    """Every rank gets the whole field's total bit for bit (the columns
    summed one after another in x order, as the single-field kernel does)
    and the maxima over the ranks."""
    import torch.multiprocessing as mp
    n = 11
    mp.spawn(_tau_rank, args=(world, _free_port(), nx, n, str(tmp_path)), nprocs=world, join=True)
    cols = np.random.default_rng(5).standard_normal((nx, n)) * 10 ** np.random.default_rng(6).uniform(-3, 3, (nx, 1))
    want = np.zeros(n)
    for c in cols:
        want = want + c
    wmax = np.max([[r + 0.5, 10.0 - r, 2.0 * r] for r in range(world)], axis=0)
    for r in range(world):
        got = np.load(os.path.join(tmp_path, "t%d.npy" % r))
        np.testing.assert_array_equal(got[:n], want)
        np.testing.assert_array_equal(got[n:], wmax)
