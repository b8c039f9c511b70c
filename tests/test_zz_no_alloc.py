"""The allocation-free entry point fz_forward_device_static.

It serves callers that may not allocate device memory while a call runs (a
host framework that owns the device allocator, real-time loops): its
scratch is a static device array instead of the context's grow-on-demand
buffers.  Its results must equal those of fz_forward_device on the same
inputs, on consecutive calls (the array keeps the previous call's contents),
and batches that do not fit the array must be rejected.

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_scratch_entry_point_matches_allocating_one(fz):
    """Both entry points launch the same kernels with the same launch shapes
    (the chemistry chain's lanes and warps come from the context in both) on
    the same inputs, so they agree bit for bit: Pg given, hydrostatic from
    the top, and hydrostatic from the log tau5 anchor (k_chain_med)."""
    import torch
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    nz, ncol = 64, 96
    ctx = fz.Synthesis(lines, reg, nz=nz)
    stream = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((21, 22)):           # two calls in a row, different inputs
        for he in (0, 1, 2):                         # FZ_HE_NONE, FZ_HE_TOP, FZ_HE_LTAU
            m = torch.from_numpy(fz.atmos.make_columns(ncol, nz, seed=seed + 10 * he)).cuda()
            syn_a = torch.zeros((ncol, 4, ctx.numw), dtype=torch.float64, device="cuda")
            syn_b = torch.full_like(syn_a, float("nan"))
            mo_a, mo_b = torch.empty_like(m), torch.empty_like(m)
            st_a = torch.zeros(ncol, dtype=torch.int32, device="cuda")
            st_b = torch.full_like(st_a, -7)
            ctx.forward_device(m.data_ptr(), ncol, syn_a.data_ptr(), mo_a.data_ptr(), st_a.data_ptr(),
                               stream=stream, hydrostatic=he)
            ctx.forward_device_static(m.data_ptr(), ncol, syn_b.data_ptr(), mo_b.data_ptr(), st_b.data_ptr(),
                                      stream=stream, hydrostatic=he)
            torch.cuda.synchronize()
            a, b = syn_a.cpu().numpy(), syn_b.cpu().numpy()
            assert np.all(st_a.cpu().numpy() == 0) and np.all(st_b.cpu().numpy() == 0), (call, he)
            assert np.all(np.isfinite(b)), (call, he)
            assert np.array_equal(a, b), (call, he, float(np.max(np.abs(a - b))))
            assert np.array_equal(mo_a.cpu().numpy(), mo_b.cpu().numpy()), (call, he)


def test_static_scratch_rejects_oversize_batches(fz):
    import torch
    lines = fz.lines_parse(fz.atmos.line_database_text())
    reg = fz.regions_from_lines_section(fz.atmos.lines_section(2), lines)
    nz, ncol = 128, 8192                              # ~100 MB of scratch > 64 MiB
    ctx = fz.Synthesis(lines, reg, nz=nz)
    m = torch.zeros((ncol, 13, nz), dtype=torch.float32, device="cuda")
    syn = torch.zeros((ncol, 4, ctx.numw), dtype=torch.float64, device="cuda")
    with pytest.raises(fz.FzError, match="size limit"):
        ctx.forward_device_static(m.data_ptr(), ncol, syn.data_ptr(), m.data_ptr())
