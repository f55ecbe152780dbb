"""The headline batch itself: 64 complex fields at lmax 1024, n = 0,
envelope (l+1)^-1.5 (the shape bench.py times), every tensor-core form
against the FP64 path on the same inputs, with the bars the metric states:
BF16x3 and the 4-slice Ozaki form <= 1e-6 (inverse and forward), Ozaki
<= 1e-12. Plus the Ozaki form on a steeper spectrum, (l+1)^-2.5, where its
one exponent per coefficient row leaves the high degrees fewer of the 49
slice bits: still within its 1e-12 bar at this size (measured 3.5e-13
inverse, 1.6e-14 forward)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu

L, B = 1024, 64


def _coefficients(torch, power, seed):
    rng = np.random.default_rng(seed)
    c = np.stack([oracle.random_coefficients(rng, L, L, 0, False, power) for _ in range(B)])
    return torch.from_numpy(c).cuda()


def _errors(g, torch, coef, prec, ref_f, ref_c):
    f = torch.empty_like(ref_f)
    g.inverse_batch(L, 0, coef, f, prec)
    c = torch.zeros_like(coef)
    g.forward_batch(L, 0, ref_f, c, prec)
    torch.cuda.synchronize()
    g.device_status()
    return (float(torch.linalg.norm(f - ref_f) / torch.linalg.norm(ref_f)),
            float(torch.linalg.norm(c - ref_c) / torch.linalg.norm(ref_c)))


def test_headline_batch_errors_against_fp64():
    import torch

    import gshtrans_b200 as gsht

    coef = _coefficients(torch, 1.5, 2024)
    with gsht.GaussLegendreGrid(L, 0, nrange=gsht.Single,
                                forms=("bf16x3", "ozaki", "ozaki4")) as g:
        ref_f = torch.empty((B, g.FieldSize()), dtype=torch.complex128, device="cuda")
        g.inverse_batch(L, 0, coef, ref_f, "fp64")
        ref_c = torch.zeros_like(coef)
        g.forward_batch(L, 0, ref_f, ref_c, "fp64")
        for prec, tol in (("bf16x3", 1e-6), ("ozaki4", 1e-6), ("ozaki", 1e-12)):
            inv, fwd = _errors(g, torch, coef, prec, ref_f, ref_c)
            assert inv < tol and fwd < tol, (prec, inv, fwd)
        # and the FP64 path's own round trip
        assert relerr(ref_c.cpu().numpy(), coef.cpu().numpy()) < 1e-12


def test_ozaki_on_a_steeper_spectrum():
    import torch

    import gshtrans_b200 as gsht

    coef = _coefficients(torch, 2.5, 77)
    with gsht.GaussLegendreGrid(L, 0, nrange=gsht.Single, forms=("ozaki",)) as g:
        ref_f = torch.empty((B, g.FieldSize()), dtype=torch.complex128, device="cuda")
        g.inverse_batch(L, 0, coef, ref_f, "fp64")
        ref_c = torch.zeros_like(coef)
        g.forward_batch(L, 0, ref_f, ref_c, "fp64")
        inv, fwd = _errors(g, torch, coef, "ozaki", ref_f, ref_c)
        assert inv < 1e-12 and fwd < 1e-12, (inv, fwd)
