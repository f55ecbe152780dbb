"""The sharded transform on the GPU: two ranks (processes) on one device,
exchanging spectra over gloo through host copies, each running the library's
stages (gsht_forward_rings / _orders, gsht_inverse_orders / _rings) on its
slab of rings and its share of orders. The slabs of the inverse and the
summed forward equal the single-process transforms of the same grid (the
same kernels per ring and per order: equal to rounding of the sums over
ranks). Ring lengths cover every FFT path: 128 (compile-time radix-8),
192 (register Stockham, radix 3), 140 (generic), 512 (three-pass)."""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import relerr
from test_sharded_host import _collect

pytestmark = pytest.mark.gpu

CASES = [(64, 1, False), (96, 0, True), (70, -1, False), (256, 2, True)]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    import gshtrans_b200 as gsht
    from gshtrans_b200.sharded import ShardedTransform

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        res = []
        for L, n, is_real in CASES:
            rng = np.random.default_rng(1000 + L)
            cnt = 3
            c = np.stack([gsht.random_coefficients(rng, L, L, n, is_real, 1.0) for _ in range(cnt)])
            with gsht.GaussLegendreGrid(L, 2) as g:
                sh = ShardedTransform(g)
                dc = torch.from_numpy(c).cuda()
                dt = torch.float64 if is_real else torch.complex128
                grid = torch.zeros((cnt, g.FieldSize()), dtype=dt, device="cuda")
                sh.inverse(L, n, is_real, cnt, dc, grid)
                whole = torch.zeros_like(grid)
                g.inverse_batch(L, n, dc, whole)
                out = torch.zeros_like(dc)
                sh.forward(L, n, is_real, cnt, whole, out)
                ref = torch.zeros_like(dc)
                g.forward_batch(L, n, whole, ref)
                torch.cuda.synchronize()
                g.device_status()
                b, e = sh.slabs[rank]
                res.append((L, is_real, grid.view(cnt, L + 1, -1)[:, b:e].cpu().numpy(),
                            whole.view(cnt, L + 1, -1)[:, b:e].cpu().numpy(),
                            out.cpu().numpy(), ref.cpu().numpy()))
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_one_gpu_match_the_single_transform():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29800 + (os.getpid() % 500)
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = _collect(q, procs, limit=600.0)
    for rank, res in out:
        for L, is_real, g_sh, g_ref, c_sh, c_ref in res:
            assert relerr(g_sh, g_ref) < 1e-15, (rank, L, is_real)
            assert relerr(c_sh, c_ref) < 1e-15, (rank, L, is_real)
