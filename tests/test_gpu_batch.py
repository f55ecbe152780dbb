"""Batched transforms of fields of uneven size (gsht_plan_batch /
gsht_batch_execute, one CUDA graph per mode) against the single-field calls
(GaussLegendreGrid.h:108-321 semantics: the forward adds into its output)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gsht():
    import gshtrans_b200

    return gshtrans_b200


def _fields(torch, rng, specs):
    out = []
    for lmax, n, is_real in specs:
        c = oracle.random_coefficients(rng, lmax, lmax, n, is_real, 1.0)
        cin = torch.from_numpy(c).cuda()
        npts = (lmax + 1) * 2 * lmax
        grid = torch.zeros(npts, dtype=torch.float64 if is_real else torch.complex128, device="cuda")
        init = rng.standard_normal(c.size) + 1j * rng.standard_normal(c.size)
        cout = torch.from_numpy(init).cuda()
        out.append((lmax, n, is_real, cin, grid, cout, init))
    return out


SPECS = [(32, 0, False), (32, 0, False), (32, -1, True), (64, 2, False), (64, 2, False),
         (64, 0, True), (128, -2, False), (128, 1, True), (128, 1, True), (128, 1, True),
         (48, 0, False), (96, -1, True)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("bf16x3", 1e-12), ("ozaki", 1e-14), ("ozaki4", 1e-14)])
def test_batch_matches_single_field_calls(gsht, precision, tol):
    import torch

    rng = np.random.default_rng(31)
    fields = _fields(torch, rng, SPECS)
    batch = gsht.Batch([f[:6] for f in fields], precision=precision, autotune=True)
    groups, grids, nodes = batch.info()
    assert grids == len({s[0] for s in SPECS})
    assert groups == len(set(SPECS))
    assert min(nodes) > 0
    for lm, n, re, cnt, tile in batch.groups():
        assert tile in (32, 64, 128)
    assert batch.streams() in (1, 2, 4, 8, 16)
    # planning (warm-up, tile-width and schedule tuning) leaves the callers'
    # buffers as they were
    torch.cuda.synchronize()
    for lmax, n, is_real, cin, grid, cout, init in fields:
        assert not torch.any(grid)
        assert np.array_equal(cout.cpu().numpy(), init)
    batch.round_trip()
    torch.cuda.synchronize()
    forms = () if precision == "fp64" else (precision,)
    for lmax, n, is_real, cin, grid, cout, init in fields:
        with gsht.GaussLegendreGrid(lmax, abs(n), forms=forms) as g:
            f1 = torch.zeros_like(grid)
            g.InverseTransformation(lmax, n, cin, f1, precision)
            c1 = torch.from_numpy(init).cuda()
            g.ForwardTransformation(lmax, n, f1, c1, precision)
            torch.cuda.synchronize()
        assert relerr(grid.cpu().numpy(), f1.cpu().numpy()) < tol, (lmax, n, is_real)
        assert relerr(cout.cpu().numpy(), c1.cpu().numpy()) < tol, (lmax, n, is_real)
    batch.close()


def test_batch_modes_and_replays(gsht):
    import torch

    rng = np.random.default_rng(7)
    fields = _fields(torch, rng, SPECS[:6])
    batch = gsht.Batch([f[:6] for f in fields], precision="fp64", autotune=False)
    batch.inverse()
    grids1 = [f[4].clone() for f in fields]
    batch.inverse()  # the inverse overwrites: same grids again
    for a, f in zip(grids1, fields):
        assert torch.equal(a, f[4])
    inits = [f[5].clone() for f in fields]
    batch.forward()
    once = [f[5].clone() - i for f, i in zip(fields, inits)]
    batch.forward()  # the forward accumulates: twice the result
    torch.cuda.synchronize()
    for o, f, i in zip(once, fields, inits):
        # complex fields: c_{L,L} is set to 0, not accumulated (GaussLegendreGrid.h:209-215)
        k = o.numel() if f[2] else o.numel() - 1
        if not f[2]:
            assert f[5][-1].item() == 0
        assert relerr((f[5] - i)[:k].cpu().numpy(), (2 * o)[:k].cpu().numpy()) < 1e-14
        # and the round trip recovers the coefficients
        assert relerr(o[:k].cpu().numpy(), f[3][:k].cpu().numpy()) < 1e-12
    batch.close()


def test_bf16x3_batch_one_legendre_launch_matches_per_group_launches(gsht, monkeypatch):
    """The BF16x3 plan runs each direction's Legendre stage as one launch over
    the work list of every group; with GSHT_BATCH_FUSED=0 each group runs
    its own transform. Same operand rows, same products in the same order per
    output element: the two agree to the last bits."""
    import torch

    rng = np.random.default_rng(11)
    specs = SPECS + [(200, 0, False), (200, 0, False), (200, 2, True)]
    fa = _fields(torch, rng, specs)
    fb = [(lm, n, re, cin, torch.zeros_like(g), torch.from_numpy(init).cuda(), init)
          for lm, n, re, cin, g, cout, init in fa]
    fused = gsht.Batch([f[:6] for f in fa], precision="bf16x3", autotune=True)
    monkeypatch.setenv("GSHT_BATCH_FUSED", "0")
    per_group = gsht.Batch([f[:6] for f in fb], precision="bf16x3", autotune=False)
    fused.round_trip()
    per_group.round_trip()
    torch.cuda.synchronize()
    for a, b in zip(fa, fb):
        assert relerr(a[4].cpu().numpy(), b[4].cpu().numpy()) < 1e-15, a[:3]
        assert relerr(a[5].cpu().numpy(), b[5].cpu().numpy()) < 1e-15, a[:3]
    tiles = {t for *_, t in fused.groups()}
    assert len(tiles) == 1 and tiles <= {32, 64, 128}  # one launch, one tile width
    fused.close()
    per_group.close()
