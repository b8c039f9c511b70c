"""A field split over ranks by x (one process per GPU), for the pieces of the
inversion that couple pixels: SMOOTHING_B at the start of every cycle
(src/model_spatial_extension.f90:351-491; its x pass reads the neighbouring
x columns) and SET_TAU's assists (src/invert3d.f90:492-727: a field sum of
Stokes I and three field maxima); the inversion itself and END_CYCLE's
synthesis are per pixel.

Rank r holds field columns [x0, x1) (a contiguous run of pixels iy + NY ix);
before smoothing, every rank sends its first and last columns to its
neighbours over torch.distributed (NCCL on the GPUs, gloo in the CPU tests)
and smooths its columns with the neighbours' halos attached; the field's own
edge and 4-point rules apply (fz_smooth_shard_device), so the result equals
the whole field's SMOOTHING_B.
"""
import numpy as np


def split(n, world):
    """[x0, x1) of every rank: near-equal contiguous runs of n columns."""
    b = [n * r // world for r in range(world + 1)]
    return [(b[r], b[r + 1]) for r in range(world)]


class FieldShard:
    """Rank `rank` of `world` holding columns split(nx_field, world)[rank] of
    an nx_field x ny field."""

    def __init__(self, nx_field, ny, rank, world, group=None):
        self.nx_field, self.ny, self.rank, self.world, self.group = int(nx_field), int(ny), rank, world, group
        self.x0, self.x1 = split(self.nx_field, world)[rank]
        self.nx = self.x1 - self.x0
        if self.nx < 1:
            raise ValueError("more ranks than field columns")

    def exchange_halo(self, local):
        """local: this rank's models (nx*ny, 13, nz) (torch, on the device of
        the process group's backend).  Returns (extended array, its first
        field column): the left neighbour's last column and the right
        neighbour's first column attached where they exist."""
        import torch
        import torch.distributed as dist
        ny = self.ny
        parts, x0 = [local], self.x0
        if self.world > 1:
            ops, recv = [], {}
            if self.rank > 0:
                recv["l"] = torch.empty_like(local[:ny])
                ops.append(dist.P2POp(dist.isend, local[:ny].contiguous(), self.rank - 1, group=self.group))
                ops.append(dist.P2POp(dist.irecv, recv["l"], self.rank - 1, group=self.group))
            if self.rank < self.world - 1:
                recv["r"] = torch.empty_like(local[:ny])
                ops.append(dist.P2POp(dist.isend, local[-ny:].contiguous(), self.rank + 1, group=self.group))
                ops.append(dist.P2POp(dist.irecv, recv["r"], self.rank + 1, group=self.group))
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            if "l" in recv:
                parts.insert(0, recv["l"])
                x0 -= 1
            if "r" in recv:
                parts.append(recv["r"])
        return torch.cat(parts, 0), x0

    def smooth(self, local, smoother, params=None):
        """SMOOTHING_B of this rank's columns, in place on local.  smoother(
        ext, nx_ext, ny, x0_ext, nx_field, params) smooths an extended array in
        place: Synthesis.smooth_shard_device on the GPU (see device_smoother)."""
        ext, x0 = self.exchange_halo(local)
        nx_ext = ext.shape[0] // self.ny
        smoother(ext, nx_ext, self.ny, x0, self.nx_field, params)
        off = (self.x0 - x0) * self.ny
        local.copy_(ext[off:off + self.nx * self.ny])

    def field_reduce(self):
        """The two field-wide reductions of SET_TAU for this rank
        (fz_set_tau_shard_device's reduce): fn(kind, data, n, nx) on a numpy
        view.  kind 0 -- data[:nx*n] holds this rank's per-column sums
        (x-major); every rank's columns are gathered in field x order and
        summed one after another (the order of the whole field's sum), the
        total left in data[:n]; kind 1 -- data[:3] becomes the maximum over
        the ranks."""
        import torch
        import torch.distributed as dist
        sizes = [x1 - x0 for x0, x1 in split(self.nx_field, self.world)]

        def device():
            if self.world == 1:
                return "cpu"
            return "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"

        def fn(kind, data, n, nx):
            if kind == 0:
                part = np.array(data[:nx * n], dtype=np.float64).reshape(nx, n)
                if self.world == 1:
                    rows = part
                else:
                    buf = torch.zeros((max(sizes), n), dtype=torch.float64, device=device())
                    buf[:nx] = torch.from_numpy(part)
                    got = [torch.empty_like(buf) for _ in range(self.world)]
                    dist.all_gather(got, buf, group=self.group)
                    rows = np.concatenate([g.cpu().numpy()[:k] for g, k in zip(got, sizes)])
                tot = np.zeros(n)
                for r in rows:
                    tot = tot + r
                data[:n] = tot
            else:
                t = torch.tensor(np.array(data[:3], dtype=np.float64), device=device())
                if self.world > 1:
                    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
                data[:3] = t.cpu().numpy()
            return 0
        return fn

    def set_tau(self, ctx, d_obs, d_models, assist, hydrostatic=True, stream=0):
        """SET_TAU's assists on this rank's pixels, the field sums and maxima
        over all ranks: equal to the whole field's fz_set_tau."""
        ctx.set_tau_shard_device(self.nx, self.ny, d_obs.data_ptr(), d_models.data_ptr(), assist,
                                 self.field_reduce(), hydrostatic=hydrostatic, stream=stream)

    def invert_cycles(self, ctx, d_obs, d_models, cycles, hydrostatic=True, opts=None, stream=0):
        """INVERT3D's cycles on this rank's pixels (d_obs (nx*ny, 4, numw)
        float64, d_models (nx*ny, 13, nz) float32, torch tensors on the GPU):
        per cycle the node layout, SMOOTHING_B across ranks, the batched
        inversion from a fresh LM state and END_CYCLE's synthesis; d_models
        holds the last cycle's models on return.  Returns (chi2, iterations,
        status) of the last cycle (device tensors)."""
        import torch
        npix = self.nx * self.ny
        best = torch.empty_like(d_models)
        syn = torch.empty((npix, 4, ctx.numw), dtype=torch.float64, device=d_models.device)
        chi = torch.empty(npix, dtype=torch.float64, device=d_models.device)
        it = torch.empty(npix, dtype=torch.int32, device=d_models.device)
        st = torch.empty(npix, dtype=torch.int32, device=d_models.device)
        smoother = device_smoother(ctx)
        assist = (opts.assist & 15) if opts is not None else 0
        for cy, nodes in enumerate(cycles):
            ctx.rf_nodes(nodes)
            torch.cuda.synchronize()
            # SET_TAU's assists when neither Pg nor P0 is free, every cycle
            # or, with PROGRESSIVE, the first (src/invert3d.f90:505-520)
            if assist and not nodes.get(2, 0) and not nodes.get(8, 0) and (cy == 0 or not opts.assist & 16):
                self.set_tau(ctx, d_obs, d_models, assist, hydrostatic=bool(hydrostatic), stream=stream)
                torch.cuda.synchronize()
            self.smooth(d_models, smoother)
            torch.cuda.synchronize()
            ctx.invert_device(npix, d_obs.data_ptr(), d_models.data_ptr(), best.data_ptr(), chi.data_ptr(),
                              it.data_ptr(), st.data_ptr(), hydrostatic=hydrostatic, opts=opts, stream=stream)
            ctx.forward_device(best.data_ptr(), npix, syn.data_ptr(), d_models.data_ptr(), 0, stream=stream,
                               hydrostatic=bool(hydrostatic))
            torch.cuda.synchronize()
        return chi, it, st


def device_smoother(ctx):
    """The GPU smoother for FieldShard.smooth: the free parameters of the
    context's node layout (or params)."""
    def f(ext, nx, ny, x0, nx_field, params):
        ctx.smooth_shard_device(ext.data_ptr(), nx, ny, x0, nx_field, params)
    return f


def host_smoother(oracle_shard_fn, params_default):
    """A CPU smoother over a numpy restatement (tests)."""
    def f(ext, nx, ny, x0, nx_field, params):
        import torch
        out = oracle_shard_fn(ext.numpy(), nx, ny, x0, nx_field, params or params_default)
        ext.copy_(torch.from_numpy(out))
    return f
