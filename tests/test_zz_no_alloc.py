"""bp_residual_noalloc: the residual entry point that allocates nothing.

It exists for callers that own all device memory themselves (a fixed pool
or budget, or code that must not hit the implicit device synchronisation of
cudaMalloc/cudaFree during a time step): they hand in their own device
buffers and the kernel keeps its reduction scratch in a fixed file-scope
device array.  This test calls it through the C ABI with device buffers
(allocated here, by the test, with torch) and checks its residual and norms
against the existing bp_matvec entry point, on two calls in a row (the
second call reuses the shared scratch left by the first).  This file is
named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from cism_b200 import configs, solver

from helpers import oracle_system, owned_active_rows, random_state

pytestmark = pytest.mark.gpu

_dp = C.c_void_p


@pytest.mark.parametrize("m", [configs.slab(n=24), configs.dome()], ids=lambda m: m.name)
def test_noalloc_residual_matches_matvec(ctx, m):
    import torch

    lib = solver.lib()
    lib.bp_residual_noalloc.argtypes = [C.c_int] * 4 + [_dp] * 13
    lib.bp_residual_noalloc.restype = C.c_int
    su, _, _, A, bu, bv, _ = oracle_system(m, seed=11)
    xu, xv = random_state(m, su, seed=12, scale=5.0)
    # expected through the existing entry point
    yu, yv = ctx.matvec(m, su["active_vertex"], A, xu, xv)
    rows = owned_active_rows(m, su["active_vertex"])
    eu = np.where(rows[..., None], yu - bu, 0.0)
    ev = np.where(rows[..., None], yv - bv, 0.0)
    enr = np.sqrt(np.sum(eu ** 2 + ev ** 2))
    enb = np.sqrt(np.sum(np.where(rows[..., None], bu ** 2 + bv ** 2, 0.0)))
    dev = torch.device("cuda:0")
    t = lambda a, dt=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
    dA = [t(a) for a in A]
    dxu, dxv, dbu, dbv = t(xu), t(xv), t(bu), t(bv)
    dav = t(su["active_vertex"], torch.int32)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        dru = torch.full(m.vshape3, np.nan, device=dev, dtype=torch.float64)
        drv = torch.full(m.vshape3, np.nan, device=dev, dtype=torch.float64)
        dn = torch.full((3,), np.nan, device=dev, dtype=torch.float64)
        rc = lib.bp_residual_noalloc(m.nx, m.ny, m.nz, m.periodic, dav.data_ptr(),
                                     *[a.data_ptr() for a in dA], dxu.data_ptr(), dxv.data_ptr(),
                                     dbu.data_ptr(), dbv.data_ptr(), dru.data_ptr(), drv.data_ptr(),
                                     dn.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize(dev)
        ru, rv, nrm = dru.cpu().numpy(), drv.cpu().numpy(), dn.cpu().numpy()
        scale = np.max(np.abs(eu)) + np.max(np.abs(ev))
        assert np.max(np.abs(ru - eu)) <= 1e-13 * scale, call
        assert np.max(np.abs(rv - ev)) <= 1e-13 * scale, call
        assert abs(nrm[0] - enr) <= 1e-13 * enr, call
        assert abs(nrm[1] - enb) <= 1e-13 * enb, call
        assert abs(nrm[2] - enr / enb) <= 1e-12 * (enr / enb), call


def test_noalloc_rejects_oversize(ctx):
    lib = solver.lib()
    lib.bp_residual_noalloc.argtypes = [C.c_int] * 4 + [_dp] * 13
    # 4100 x 4100 x 1 rows exceed the fixed scratch; rejected before any launch
    one = C.c_void_p(1)
    rc = lib.bp_residual_noalloc(4101, 4101, 1, 1, *([one] * 12), None)
    assert rc == 10
