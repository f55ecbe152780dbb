"""Canonical-component expansions wired to the transforms (the reference
declares CanonicalComponentExpansion, CanonicalComponentExpansion.h:36-105,
but never connects it to the grid).

Bars: the packed (l, m) index agrees with GSHIndices (Indexing.h:104-131);
to_field / from_field give exactly what the grid's own transform calls give;
coefficients -> field -> coefficients is the identity to 1e-12 (the
reference's round-trip bar, tests/CheckCoeff2Coeff.h:40-84)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    import gshtrans_b200
    from gshtrans_b200 import expansions, fields

    return gshtrans_b200, expansions, fields


@pytest.mark.parametrize("n,is_real", [(0, False), (-2, False), (1, True)])
def test_index_matches_the_packed_layout(mods, n, is_real):
    gsht, E, _ = mods
    with gsht.GaussLegendreGrid(24, 2) as g:
        e = E.Expansion(g, n, is_real)
        ls, ms = gsht.degree_order(24, n, is_real)
        assert e.Size() == ls.size
        assert [e.Index(int(l), int(m)) for l, m in zip(ls, ms)] == list(range(ls.size))
        with pytest.raises(gsht.BadArgument):
            e.Index(abs(n) - 1, 0) if n else e.Index(25, 0)


@pytest.mark.parametrize("is_real", [False, True])
def test_round_trips_and_parity_with_the_grid_calls(mods, is_real):
    import torch

    gsht, E, F = mods
    L, n = 96, 1
    rng = np.random.default_rng(11 + is_real)
    with gsht.GaussLegendreGrid(L, 1) as g:
        c = oracle.random_coefficients(rng, L, L, n, is_real)
        e = E.Expansion(g, n, is_real, data=torch.from_numpy(c).cuda())
        f = e.to_field()
        direct = np.zeros(g.FieldSize(), np.float64 if is_real else np.complex128)
        g.InverseTransformation(L, n, c, direct)
        assert np.array_equal(f.Data().cpu().numpy(), direct)
        back = E.Expansion.of(f)
        assert relerr(back.Data().cpu().numpy(), c) < 1e-12
        out = np.zeros_like(c)
        g.ForwardTransformation(L, n, direct, out)
        assert np.array_equal(back.Data().cpu().numpy(), out)
        # from_field replaces (does not add to) what the expansion held
        back.from_field(f)
        assert relerr(back.Data().cpu().numpy(), c) < 1e-12
        # element access by (l, m)
        assert back[L - 1, 2] == pytest.approx(complex(c[back.Index(L - 1, 2)]), abs=1e-12)
        back[n + 3, 0] = 5.0
        assert back[n + 3, 0] == 5.0


def test_batches_partial_degree_and_compound_operators(mods):
    import torch

    gsht, E, F = mods
    L, lmax, n, B = 64, 40, -1, 3
    rng = np.random.default_rng(5)
    with gsht.GaussLegendreGrid(L, 1) as g:
        cs = np.stack([oracle.random_coefficients(rng, L, lmax, n, False) for _ in range(B)])
        e = E.Expansion(g, n, count=B, lmax=lmax, data=torch.from_numpy(cs).cuda())
        f = e.to_field(precision="fp64")
        for b in range(B):
            single = E.Expansion(g, n, lmax=lmax, data=torch.from_numpy(cs[b]).cuda()).to_field()
            assert relerr(f.Data()[b].cpu().numpy(), single.Data().cpu().numpy()) < 1e-14
        back = E.Expansion.of(f, lmax=lmax)
        assert relerr(back.Data().cpu().numpy(), cs) < 1e-12
        back -= e
        assert float(back.Data().abs().max()) < 1e-12
        back.assign(e)
        back *= 2.0
        back += e
        back /= 3.0
        assert relerr(back.Data().cpu().numpy(), cs) < 1e-15
        with pytest.raises(gsht.BadArgument):
            back += E.Expansion(g, n, lmax=lmax)  # batch sizes differ
        with pytest.raises(gsht.BadArgument):
            E.Expansion(g, n).from_field(F.Field(g, 0))  # upper indices differ


def test_tensor_core_precisions(mods):
    import torch

    gsht, E, _ = mods
    L, n = 128, 0
    rng = np.random.default_rng(3)
    with gsht.GaussLegendreGrid(L, 0, forms=("bf16x3", "ozaki")) as g:
        c = oracle.random_coefficients(rng, L, L, n, False, 1.0)
        e = E.Expansion(g, n, data=torch.from_numpy(c).cuda())
        for prec, tol in (("bf16x3", 2e-6), ("ozaki", 1e-12)):
            back = E.Expansion.of(e.to_field(precision=prec), precision=prec)
            assert relerr(back.Data().cpu().numpy(), c) < tol, prec
