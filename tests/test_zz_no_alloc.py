"""gsht_inverse_noalloc: the allocation-free FP64 inverse transform.

It exists for callers that may not allocate device memory when they
transform (an arena or caching allocator owns the device, a latency-critical
loop cannot take an allocation's implicit synchronisation, or start-up must
be the last place an out-of-memory error can happen). Its scratch is a fixed
array in the library's device memory, so its output must equal the
allocating entry point's on every call, including consecutive calls that
reuse the same scratch. This file is collected last on purpose.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the FP64 path's tolerance


def _entry(lib):
    f = lib.gsht_inverse_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_noalloc_inverse_matches_gsht_inverse_on_consecutive_calls():
    import torch

    import gshtrans_b200 as gsht

    noalloc = _entry(gsht.library)
    rng = np.random.default_rng(4242)
    for L, n, lmax in ((96, -2, 96), (256, 1, 200)):
        with gsht.GaussLegendreGrid(L, 2) as g:
            for is_real in (False, True):
                for call in range(2):  # two calls in a row share the scratch
                    c = oracle.random_coefficients(rng, L, lmax, n, is_real, 1.0)
                    dc = torch.from_numpy(c).cuda()
                    dt = torch.float64 if is_real else torch.complex128
                    want = torch.zeros(g.FieldSize(), dtype=dt, device="cuda")
                    g.InverseTransformation(lmax, n, dc, want)  # existing entry point
                    got = torch.full((g.FieldSize(),), float("nan"), dtype=dt, device="cuda")
                    st = noalloc(g._h, lmax, n, int(is_real), dc.data_ptr(), got.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream)
                    assert st == 0, gsht.library.gsht_last_error()
                    torch.cuda.synchronize()
                    g.device_status()
                    assert relerr(got.cpu().numpy(), want.cpu().numpy()) < TOL, (L, is_real, call)


def test_noalloc_rejects_sizes_beyond_its_scratch_and_host_pointers():
    import torch

    import gshtrans_b200 as gsht

    noalloc = _entry(gsht.library)
    with gsht.GaussLegendreGrid(1024, 0, nrange=gsht.Single) as g:
        c = torch.zeros(gsht.coefficient_size(1024, 0, False), dtype=torch.complex128, device="cuda")
        f = torch.zeros(g.FieldSize(), dtype=torch.complex128, device="cuda")
        st = noalloc(g._h, 1024, 0, 0, c.data_ptr(), f.data_ptr(), None)
        assert st == 5 and b"bytes of scratch" in gsht.library.gsht_last_error()
        h = np.zeros(gsht.coefficient_size(64, 0, False), np.complex128)
        st = noalloc(g._h, 64, 0, 0, h.ctypes.data, f.data_ptr(), None)
        assert st == 1


def test_noalloc_makes_no_device_allocation_on_a_fresh_grid():
    # Called first on a grid no other transform has touched (no operand
    # layout or workspace cached), then three times more: the library's own
    # allocation counter does not move, and after the first call (which on a
    # fresh process loads the library's device module and with it the
    # 16 MiB array) the device's free memory does not change either.
    import torch

    import gshtrans_b200 as gsht

    noalloc = _entry(gsht.library)
    rng = np.random.default_rng(77)
    L, n = 128, 1
    with gsht.GaussLegendreGrid(L, 1) as g:
        c = oracle.random_coefficients(rng, L, L, n, False, 1.0)
        dc = torch.from_numpy(c).cuda()
        outs = [torch.zeros(g.FieldSize(), dtype=torch.complex128, device="cuda") for _ in range(4)]
        torch.cuda.synchronize()
        stats0 = gsht.alloc_stats()
        s = torch.cuda.current_stream().cuda_stream
        assert noalloc(g._h, L, n, 0, dc.data_ptr(), outs[0].data_ptr(), s) == 0
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for k in range(1, 4):
            assert noalloc(g._h, L, n, 0, dc.data_ptr(), outs[k].data_ptr(), s) == 0
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        assert gsht.alloc_stats() == stats0
        g.device_status()
        want = torch.zeros_like(outs[0])
        g.InverseTransformation(L, n, dc, want)
        for k in range(4):
            assert relerr(outs[k].cpu().numpy(), want.cpu().numpy()) < TOL
