"""The sharded transform's exchange logic (gshtrans_b200.sharded) on CPU:
world size 2 and 3 over gloo, with the stages restated on the oracle
(tests/sharded_stages.py). Every rank's slab of an inverse and the summed
forward equal the oracle's whole transforms (GaussLegendreGrid.h:108-321)."""

from __future__ import annotations

import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import relerr


def _collect(q, procs, limit=300.0):
    """The ranks' results; fails as soon as a rank exits without one."""
    import queue
    import time

    out, t0 = [], time.time()
    while len(out) < len(procs):
        try:
            out.append(q.get(timeout=2.0))
        except queue.Empty:
            bad = [p.exitcode for p in procs if p.exitcode not in (None, 0)]
            assert not bad, f"a rank failed (exit codes {bad})"
            assert time.time() - t0 < limit, "ranks did not report in time"
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def _worker(rank, world, port, L, n, q):
    import torch
    import torch.distributed as dist

    import oracle
    from gshtrans_b200.sharded import ShardedTransform
    from sharded_stages import OracleStages

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        st = OracleStages(L, n)
        sh = ShardedTransform(stages=st, n_theta=L + 1, L=L)
        res = {}
        for is_real in (False, True):
            rng = np.random.default_rng(11 + int(is_real))
            c = np.stack([oracle.random_coefficients(rng, L, L, n, is_real, 1.0) for _ in range(2)])
            grid = torch.zeros((2, (L + 1) * 2 * L), dtype=torch.float64 if is_real else torch.complex128)
            sh.inverse(L, n, is_real, 2, torch.from_numpy(c), grid)
            b, e = sh.slabs[rank]
            g = grid.numpy().reshape(2, L + 1, 2 * L)[:, b:e]
            # the forward of the oracle's whole inverse, added into a base
            whole = np.stack([st.R.inverse(L, L, n, is_real, c[f]) for f in range(2)])
            base = rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)
            out = torch.from_numpy(base.copy())
            sh.forward(L, n, is_real, 2, torch.from_numpy(whole), out)
            res[is_real] = (b, e, g, out.numpy(), whole, base, c)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_exchange_matches_the_whole_transform(world, restated):
    L, n = 12, 1
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + world * 7 + (os.getpid() % 500)
    procs = [ctx.Process(target=_worker, args=(r, world, port, L, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = _collect(q, procs)
    covered = {False: [], True: []}
    for rank, res in out:
        for is_real, (b, e, g, fwd, whole, base, c) in res.items():
            w = whole.reshape(2, L + 1, 2 * L)[:, b:e]
            if e > b:
                assert relerr(g, w) < 1e-13, (rank, is_real)
            covered[is_real].append((b, e))
            want = base + np.stack([restated.forward(L, L, n, is_real, whole[f]) for f in range(2)])
            if not is_real:
                want[:, -1] = 0  # c_{L,L} = 0 (GaussLegendreGrid.h:209-215)
            assert relerr(fwd, want) < 1e-13, (rank, is_real)
    for is_real, slabs in covered.items():
        assert sorted(slabs)[0][0] == 0 and sorted(slabs)[-1][1] == L + 1
        assert sum(e - b for b, e in slabs) == L + 1


def test_order_shares_balance_the_degrees():
    from gshtrans_b200.sharded import order_shares, ring_slabs

    for lmax, n, world in ((1024, 0, 4), (2048, 1, 8), (10, 2, 3), (5, 0, 8)):
        sh = order_shares(lmax, n, world)
        assert sh[0][0] == 0 and sh[-1][1] == lmax + 1
        assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
        work = [sum(lmax - max(m, abs(n)) + 1 for m in range(b, e)) for b, e in sh]
        if lmax >= 100:
            assert max(work) - min(work) <= lmax + 1
    sl = ring_slabs(1025, 4)
    assert sl[0][0] == 0 and sl[-1][1] == 1025 and max(e - b for b, e in sl) - min(e - b for b, e in sl) <= 1
