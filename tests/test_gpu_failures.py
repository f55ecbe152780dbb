"""Failure paths, exercised without any GPU fault, trap or hang.

Device side: every wait of the tensor-core pipelines is bounded; a wait that
runs out raises the grid's device error word and returns, and
gsht_device_status reports GSHT_ERR_TIMEOUT. gsht_check_bounded_wait makes
one such wait run out on purpose (an mbarrier phase nothing completes).

Host side: every device allocation of the library goes through one
allocator (gsht_set_allocator); a hook that refuses the k-th allocation
stands in for an out-of-memory device. The call that needed the memory must
return GSHT_ERR_OOM and give back everything it had taken, and the library
must work normally afterwards. The reference has neither path (it asserts,
GaussLegendreGrid.h:41-44, and its tables are host vectors).
"""

from __future__ import annotations

import time

import numpy as np
import pytest

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu

OOM, TIMEOUT = 2, 4


@pytest.fixture(scope="module")
def gsht():
    import gshtrans_b200

    return gshtrans_b200


class Tracker:
    """Allocation hook over PyTorch's caching allocator that counts calls,
    tracks what is live and refuses the call with index ``fail_at``."""

    def __init__(self, fail_at=None):
        self.fail_at = fail_at
        self.calls = 0
        self.live = {}

    def alloc(self, nbytes):
        import torch

        k = self.calls
        self.calls += 1
        if k == self.fail_at:
            return 0
        p = torch.cuda.caching_allocator_alloc(nbytes)
        self.live[p] = nbytes
        return p

    def free(self, p):
        import torch

        del self.live[p]
        torch.cuda.caching_allocator_delete(p)


def _round_trip_ok(gsht, g, restated, L, n, seed):
    rng = np.random.default_rng(seed)
    c = oracle.random_coefficients(rng, L, L, n, False, 1.0)
    f = np.zeros(g.FieldSize(), np.complex128)
    g.InverseTransformation(L, n, c, f)
    assert relerr(f, restated.inverse(L, L, n, False, c)) < 1e-13


def test_bounded_wait_runs_out_and_reports_timeout(gsht, restated):
    with gsht.GaussLegendreGrid(32, 0) as g:
        t0 = time.perf_counter()
        g.check_bounded_wait()
        with pytest.raises(gsht.GSHTError) as e:
            g.device_status()
        waited = time.perf_counter() - t0
        assert e.value.status == TIMEOUT and "code 100" in str(e.value)
        assert waited < 30.0
        g.device_status()  # the word was cleared by the report
        # the context is still usable
        _round_trip_ok(gsht, g, restated, 32, 0, 1)


def test_timeout_of_one_grid_leaves_other_grids_alone(gsht, restated):
    with gsht.GaussLegendreGrid(24, 1) as a, gsht.GaussLegendreGrid(24, 1) as b:
        a.check_bounded_wait()
        b.device_status()
        with pytest.raises(gsht.GSHTError):
            a.device_status()
        _round_trip_ok(gsht, b, restated, 24, 1, 2)


def test_failed_grid_allocation_reports_oom_and_releases_everything(gsht, restated):
    forms = ("bf16x3", "ozaki", "recurrence")
    probe = Tracker()
    gsht.set_allocator(probe.alloc, probe.free)
    try:
        g = gsht.GaussLegendreGrid(48, 2, forms=forms)
    finally:
        gsht.set_allocator()
    g.close()  # released through the hook that made the memory
    total = probe.calls
    assert total > 4 and not probe.live
    for k in sorted({0, 1, 2, total // 2, total - 1}):
        t = Tracker(fail_at=k)
        gsht.set_allocator(t.alloc, t.free)
        try:
            with pytest.raises(gsht.GSHTError) as e:
                gsht.GaussLegendreGrid(48, 2, forms=forms)
        finally:
            gsht.set_allocator()
        assert e.value.status == OOM, (k, str(e.value))
        assert not t.live, (k, t.live)
    a0, r0, live0 = gsht.alloc_stats()
    with gsht.GaussLegendreGrid(48, 2, forms=forms) as g:
        _round_trip_ok(gsht, g, restated, 48, 2, 3)
    a1, r1, live1 = gsht.alloc_stats()
    assert a1 - a0 == r1 - r0 and live1 == live0


def test_failed_workspace_allocation_leaves_the_grid_usable(gsht, restated):
    import torch

    L = 64
    with gsht.GaussLegendreGrid(L, 0, nrange=gsht.Single) as g:
        _round_trip_ok(gsht, g, restated, L, 0, 4)  # one field's workspace
        B = 8  # a batch needs a larger workspace: refuse it
        rng = np.random.default_rng(5)
        c = torch.from_numpy(np.stack([oracle.random_coefficients(rng, L, L, 0, False, 1.0)
                                       for _ in range(B)])).cuda()
        f = torch.zeros((B, g.FieldSize()), dtype=torch.complex128, device="cuda")
        t = Tracker(fail_at=0)
        gsht.set_allocator(t.alloc, t.free)
        try:
            with pytest.raises(gsht.GSHTError) as e:
                g.inverse_batch(L, 0, c, f)
        finally:
            gsht.set_allocator()
        assert e.value.status == OOM
        g.inverse_batch(L, 0, c, f)  # with memory available again it runs
        torch.cuda.synchronize()
        want = np.stack([restated.inverse(L, L, 0, False, c[i].cpu().numpy()) for i in range(B)])
        assert relerr(f.cpu().numpy(), want) < 1e-13


def test_torch_allocator_serves_the_library(gsht, restated):
    a0, r0, _ = gsht.alloc_stats()
    gsht.use_torch_allocator()
    try:
        with gsht.GaussLegendreGrid(40, 1, forms=("bf16x3",)) as g:
            _round_trip_ok(gsht, g, restated, 40, 1, 6)
    finally:
        gsht.set_allocator()
    a1, r1, _ = gsht.alloc_stats()
    assert a1 > a0 and a1 - a0 == r1 - r0


def test_misaligned_device_buffers_are_refused(gsht):
    """Device buffers are read as 16-byte complex elements: a buffer 8 bytes
    off that boundary is refused with GSHT_ERR_BAD_ARG before any launch."""
    import ctypes

    import torch

    from gshtrans_b200 import library
    from gshtrans_b200 import sharded  # noqa: F401  (declares the stage entry points)

    L, BAD = 32, 1
    with gsht.GaussLegendreGrid(L, 0) as g:
        cs = gsht.coefficient_size(L, 0, False)
        c = torch.zeros(2 * cs + 2, dtype=torch.float64, device="cuda")
        f = torch.zeros(2 * g.FieldSize() + 2, dtype=torch.float64, device="cuda")
        bad_c, bad_f = c.data_ptr() + 8, f.data_ptr() + 8
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert library.gsht_inverse(g._h, L, 0, 0, 0, bad_c, f.data_ptr(), s) == BAD
        assert library.gsht_inverse(g._h, L, 0, 0, 0, c.data_ptr(), bad_f, s) == BAD
        assert library.gsht_forward(g._h, L, 0, 0, 0, bad_f, c.data_ptr(), s) == BAD
        spec = torch.zeros(1 << 20, dtype=torch.float64, device="cuda")
        assert library.gsht_inverse_orders(g._h, L, 0, 0, 1, 0, L + 1, bad_c, spec.data_ptr(),
                                           s) == BAD
        # aligned buffers still run
        assert library.gsht_inverse(g._h, L, 0, 0, 0, c.data_ptr(), f.data_ptr(), s) == 0
        torch.cuda.synchronize()
        g.device_status()
