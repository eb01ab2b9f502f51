"""vfv_ilu0_apply_device_noalloc: the ILU(0) apply for callers that may not allocate device memory
while they run (fixed memory budgets, host allocators that own the device, no mid-step
cudaMalloc/cudaFree synchronisation). It takes its work vector from a fixed array inside the
library instead of allocating one, so it must give the allocating entry point's result exactly,
call after call, although every call reuses the same array.

Collected last (file name) so that a run stopping at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the bar of the other ILU(0) parity tests


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("order", [0, 1])
def test_noalloc_apply_matches_allocating_apply(gpu_ctx, c1h_system, c1_hetero, order):
    import torch
    from vfvchem_vfvm3d_b200 import Pattern, _lib
    lib = _lib.load()
    (rp, ci, va), _, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    n = c1_hetero.n
    rng = np.random.default_rng(21 + order)
    r1 = torch.tensor(rng.standard_normal(n), device="cuda")
    r2 = torch.tensor(rng.standard_normal(n), device="cuda")
    z_ref1, z_ref2, z1, z2 = (torch.empty_like(r1) for _ in range(4))
    torch.cuda.synchronize()
    lev = C.c_int32()
    # the allocating entry point: also sets up the pattern's ILU(0) storage
    for r, z in ((r1, z_ref1), (r2, z_ref2)):
        assert lib.vfv_ilu0_apply_device(gpu_ctx.handle, p.handle, order, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()), C.byref(lev)) == 0
    # two calls in a row through the no-allocation entry point (the second reuses the array the first left behind)
    for r, z in ((r1, z1), (r2, z2)):
        rc = lib.vfv_ilu0_apply_device_noalloc(gpu_ctx.handle, p.handle, order, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()),
                                               C.byref(lev))
        assert rc == 0, lib.vfv_last_error(gpu_ctx.handle)
    assert _rel(z1.cpu().numpy(), z_ref1.cpu().numpy()) <= RTOL
    assert _rel(z2.cpu().numpy(), z_ref2.cpu().numpy()) <= RTOL


def test_noalloc_rejects_unprepared_and_oversized(gpu_ctx, c1h_system, c1_hetero):
    import torch
    from vfvchem_vfvm3d_b200 import Pattern, _lib
    lib = _lib.load()
    (rp, ci, va), _, _ = c1h_system
    p = Pattern.from_csr(gpu_ctx, rp.astype(np.int32), ci)
    p.set_values(va)
    r = torch.zeros(c1_hetero.n, dtype=torch.float64, device="cuda")
    z = torch.empty_like(r)
    torch.cuda.synchronize()
    rc = lib.vfv_ilu0_apply_device_noalloc(gpu_ctx.handle, p.handle, 0, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()), None)
    assert rc == _lib.VFV_BAD_INPUT and b"not set up" in lib.vfv_last_error(gpu_ctx.handle)
    # a pattern larger than the fixed array (262,144 rows) is refused before any device work
    n = (1 << 18) + 1
    rowptr = np.arange(n + 1, dtype=np.int32)
    colind = np.arange(n, dtype=np.int32)
    big = Pattern.from_csr(gpu_ctx, rowptr, colind)
    rc = lib.vfv_ilu0_apply_device_noalloc(gpu_ctx.handle, big.handle, 0, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()), None)
    assert rc == _lib.VFV_BAD_INPUT and b"exceed" in lib.vfv_last_error(gpu_ctx.handle)


def test_noalloc_at_its_row_limit_matches_and_allocates_nothing(gpu_ctx):
    """A tridiagonal system of exactly 262,144 rows (the fixed array's size) is accepted and gives
    the allocating entry point's result; many back-to-back calls leave the device's free memory
    unchanged (nothing is allocated or freed)."""
    import torch
    from vfvchem_vfvm3d_b200 import Pattern, _lib
    lib = _lib.load()
    n = 1 << 18
    rows = [np.arange(n), np.arange(1, n), np.arange(n - 1)]
    cols = [np.arange(n), np.arange(n - 1), np.arange(1, n)]
    r_all, c_all = np.concatenate(rows), np.concatenate(cols)
    o = np.lexsort((c_all, r_all))
    r_all, c_all = r_all[o], c_all[o]
    rowptr = np.zeros(n + 1, np.int32)
    np.add.at(rowptr, r_all + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    rng = np.random.default_rng(5)
    vals = np.where(r_all == c_all, 4.0, -1.0) + 0.1 * rng.uniform(-1, 1, r_all.size)
    p = Pattern.from_csr(gpu_ctx, rowptr, c_all.astype(np.int32))
    p.set_values(vals)
    r = torch.tensor(rng.standard_normal(n), device="cuda")
    z_ref, z = torch.empty_like(r), torch.empty_like(r)
    torch.cuda.synchronize()
    lev = C.c_int32()
    assert lib.vfv_ilu0_apply_device(gpu_ctx.handle, p.handle, 0, C.c_void_p(r.data_ptr()), C.c_void_p(z_ref.data_ptr()), C.byref(lev)) == 0
    rc = lib.vfv_ilu0_apply_device_noalloc(gpu_ctx.handle, p.handle, 0, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()), C.byref(lev))
    assert rc == 0, lib.vfv_last_error(gpu_ctx.handle)
    assert _rel(z.cpu().numpy(), z_ref.cpu().numpy()) <= RTOL
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(50):
        rc = lib.vfv_ilu0_apply_device_noalloc(gpu_ctx.handle, p.handle, 0, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr()), None)
        assert rc == 0
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert _rel(z.cpu().numpy(), z_ref.cpu().numpy()) <= RTOL
