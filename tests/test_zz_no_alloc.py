"""qlgpu_rhs_noalloc: the model right-hand side for callers that cannot
allocate device memory while they run (a pre-sized device pool or arena, a
host framework that owns every device buffer, loops that cannot afford an
allocation or the synchronisation of cudaFree).  The entry point works in one
fixed scratch array inside the library; this test checks it against the
allocating entry point (qlgpu_rhs) on two calls in a row with different
inputs, so a second call cannot pass on leftovers of the first.

Kept in a file that sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

from gpu_util import rel, require_gpu
from ql_dns_b200 import _capi
from ql_dns_b200.initial import initial_state
from ql_dns_b200.params import mri_16x16_nz32
from ql_dns_b200.solver import QLSolver

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("model,NZ", [(0, 32), (1, 64)])
def test_rhs_noalloc_matches_rhs_twice(model, NZ):
    require_gpu()
    import torch
    p = mri_16x16_nz32(nx=16, ny=16, NZ=NZ, model=model, B0z=0.03 if model else 0.0, omega=0.9)
    L = _capi.load()
    cp = _capi.to_c(p)
    with QLSolver(p) as s:
        for call, (seed, t, dtl) in enumerate([(31, 0.417, 0.0021), (32, 1.093, 0.0007)]):
            lin, mf, kx0 = initial_state(p, seed, sigma=0.4, mean_u=0.02)
            s.set_state(0.0, lin, mf, kx0)
            F, Fm, Lop = s.rhs(t, dtl, lin, mf)
            d_lin, d_mf, d_kx0 = _dev(lin), _dev(mf), _dev(kx0)
            d_F = torch.empty_like(d_lin)
            d_Fm = torch.empty_like(d_mf)
            d_L = torch.empty(lin.shape, dtype=torch.float64, device="cuda")
            stream = torch.cuda.current_stream().cuda_stream
            rc = L.qlgpu_rhs_noalloc(ctypes.byref(cp), t, dtl, d_lin.data_ptr(), d_mf.data_ptr(),
                                     d_kx0.data_ptr(), d_F.data_ptr(), d_Fm.data_ptr(), d_L.data_ptr(),
                                     ctypes.c_void_p(stream))
            _capi.check(rc, None)
            torch.cuda.synchronize()
            F2, Fm2, L2 = d_F.cpu().numpy(), d_Fm.cpu().numpy(), d_L.cpu().numpy()
            assert rel(F2, F) < 1e-12, (call, rel(F2, F))
            assert rel(Fm2, Fm) < 1e-11, (call, rel(Fm2, Fm))
            assert rel(L2, Lop) < 1e-15, (call, rel(L2, Lop))


def test_rhs_noalloc_rejects_oversized_case():
    require_gpu()
    import torch
    p = mri_16x16_nz32(nx=256, ny=256, NZ=32)  # 255*128 modes > 8192: rejected before any device work
    L = _capi.load()
    cp = _capi.to_c(p)
    small = torch.zeros(16, dtype=torch.float64, device="cuda")
    ptr = ctypes.c_void_p(small.data_ptr())
    rc = L.qlgpu_rhs_noalloc(ctypes.byref(cp), 0.0, 0.0, ptr, ptr, None, ptr, ptr, None, None)
    assert rc == 1
    buf = ctypes.create_string_buffer(256)
    L.qlgpu_last_error(None, buf, 256)
    assert b"8192" in buf.value


def test_rhs_noalloc_large_grid_matches_oracle_and_changes_grid():
    # Three calls in a row on different grids: 64x64 modes at NZ = 128 (126 CTAs, so the
    # two-level reduction over CTA groups runs), then 16x16 at NZ = 32 with kx0 = NULL (the
    # library's own kx table) on the legacy default stream, then the large grid again.  A
    # table left over from the previous call would fail the next comparison.  Each result is
    # checked against the CPU oracle and against qlgpu_rhs.
    require_gpu()
    import torch
    from oracle import oracle as O
    L = _capi.load()
    big = mri_16x16_nz32(nx=64, ny=64, NZ=128)
    small = mri_16x16_nz32(nx=16, ny=16, NZ=32)
    for call, (p, seed, t, dtl, own_kx) in enumerate([(big, 41, 0.61, 0.0013, True), (small, 42, 0.29, 0.004, False),
                                                      (big, 43, 1.37, 0.0009, True)]):
        cp = _capi.to_c(p)
        lin, mf, kx0 = initial_state(p, seed, sigma=0.3)
        if own_kx:
            kx0 = kx0 + 0.25 * (2 * np.pi / p.L[0])  # a sheared wavenumber set, not the default table
        Fo, Fmo, Lo = O.rhs(p, t, dtl, lin, mf, kx0 if own_kx else None)
        with QLSolver(p) as s:
            s.set_state(0.0, lin, mf, kx0 if own_kx else None)
            F, Fm, Lop = s.rhs(t, dtl, lin, mf)
        d_lin, d_mf = _dev(lin), _dev(mf)
        d_kx0 = _dev(kx0) if own_kx else None
        d_F = torch.empty_like(d_lin)
        d_Fm = torch.empty_like(d_mf)
        d_L = torch.empty(lin.shape, dtype=torch.float64, device="cuda")
        if own_kx:
            stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        else:
            torch.cuda.synchronize()
            stream = None  # legacy default stream
        rc = L.qlgpu_rhs_noalloc(ctypes.byref(cp), t, dtl, d_lin.data_ptr(), d_mf.data_ptr(),
                                 d_kx0.data_ptr() if own_kx else None, d_F.data_ptr(), d_Fm.data_ptr(),
                                 d_L.data_ptr(), stream)
        _capi.check(rc, None)
        torch.cuda.synchronize()
        F2, Fm2, L2 = d_F.cpu().numpy(), d_Fm.cpu().numpy(), d_L.cpu().numpy()
        assert rel(F2, Fo) < 1e-11 and rel(Fm2, Fmo) < 1e-10 and rel(L2, Lo) < 1e-14, (call, rel(F2, Fo), rel(Fm2, Fmo))
        assert rel(F2, F) < 1e-12 and rel(Fm2, Fm) < 1e-11 and rel(L2, Lop) < 1e-15, call
