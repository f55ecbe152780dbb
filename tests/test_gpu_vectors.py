"""Vector fields in canonical components (gshtrans_b200.vectors) on the GPU.

Component algebra against numpy on the same component data, the pointwise
InnerProduct / DualityProduct against the reference's formulas
(VectorFieldOverloads.h:240-288), and the three-component transforms
against single-component calls and the expansion -> field -> expansion
identity (the round trip of CheckCoeff2Coeff.h, per component).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    import gshtrans_b200 as g
    from gshtrans_b200 import fields as F
    from gshtrans_b200 import vectors as V

    return g, F, V


def _random_vector(torch, V, grid, count, rng):
    u = V.VectorField(grid, count)
    shape = tuple(u.Data().shape)
    u.Data().copy_(torch.from_numpy(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)))
    return u


def test_component_algebra_and_products(mods):
    import torch

    g, F, V = mods
    rng = np.random.default_rng(3)
    with g.GaussLegendreGrid(24, 1) as grid:
        u = _random_vector(torch, V, grid, 2, rng)
        v = _random_vector(torch, V, grid, 2, rng)
        s = F.Field(grid, 0, False, 2)
        s.Data().copy_(torch.from_numpy(rng.standard_normal(tuple(s.Data().shape)) + 1.5))
        U, W, S = u.Data().cpu().numpy(), v.Data().cpu().numpy(), s.Data().cpu().numpy()
        assert [u[a].UpperIndex() for a in V.VectorField.CanonicalIndices()] == [-1, 0, 1]
        np.testing.assert_allclose((u + v).Data().cpu().numpy(), U + W, rtol=0, atol=1e-15)
        np.testing.assert_allclose((u - v).Data().cpu().numpy(), U - W, rtol=0, atol=1e-15)
        np.testing.assert_allclose((-u).Data().cpu().numpy(), -U, rtol=0, atol=0)
        np.testing.assert_allclose((u * 2.5j).Data().cpu().numpy(), U * 2.5j, rtol=1e-15)
        np.testing.assert_allclose((u * s).Data().cpu().numpy(), U * S[None], rtol=1e-15)
        np.testing.assert_allclose((u / s).Data().cpu().numpy(), U / S[None], rtol=1e-14)
        np.testing.assert_allclose(V.conj(u).Data().cpu().numpy(), np.conj(U), rtol=0, atol=0)
        w = V.VectorField(grid, 2)
        w.assign(u)
        w += v
        w *= s
        np.testing.assert_allclose(w.Data().cpu().numpy(), (U + W) * S[None], rtol=1e-14)
        w -= v
        w /= 2.0
        np.testing.assert_allclose(w.Data().cpu().numpy(), ((U + W) * S[None] - W) / 2, rtol=1e-14)
        ip = V.InnerProduct(u, v)
        assert ip.UpperIndex() == 0
        np.testing.assert_allclose(ip.Data().cpu().numpy(), np.sum(np.conj(U) * W, axis=0),
                                   rtol=1e-14, atol=1e-14)
        dp = V.DualityProduct(u, v)
        ref = -U[0] * W[2] + U[1] * W[1] - U[2] * W[0]
        np.testing.assert_allclose(dp.Data().cpu().numpy(), ref, rtol=1e-14, atol=1e-14)
        # |u|^2 = InnerProduct(u, u) is real and non-negative
        nn = V.InnerProduct(u, u).Data().cpu().numpy()
        assert np.all(np.abs(nn.imag) <= 1e-13 * np.abs(nn.real)) and np.all(nn.real > 0)


def test_component_checks(mods):
    import torch

    g, F, V = mods
    with g.GaussLegendreGrid(16, 1) as grid, g.GaussLegendreGrid(16, 1) as other, \
            g.GaussLegendreGrid(16, 0) as scalar_only:
        u = V.VectorField(grid)
        with pytest.raises(g.BadArgument):
            u[2]
        with pytest.raises(g.BadArgument):
            u + V.VectorField(other)
        with pytest.raises(g.BadArgument):
            u * F.Field(grid, 1)  # scalar fields scale with upper index 0 only
        with pytest.raises(g.BadArgument):
            V.VectorField(scalar_only)
        with pytest.raises(g.BadArgument):
            V.VectorField(grid, 2, data=torch.zeros(5, dtype=torch.complex128, device="cuda"))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("ozaki", 1e-12), ("bf16x3", 3e-6)])
def test_vector_expansion_round_trip(mods, precision, tol):
    import torch

    g, F, V = mods
    L, count = 96, 3
    rng = np.random.default_rng(11)
    forms = () if precision == "fp64" else (precision,)
    with g.GaussLegendreGrid(L, 1, forms=forms) as grid:
        e = V.VectorExpansion(grid, count)
        for a in V.VectorExpansion.CanonicalIndices():
            c = np.stack([oracle.random_coefficients(rng, L, L, a, False, 1.0) for _ in range(count)])
            e[a].Data().copy_(torch.from_numpy(c))
        u = e.to_field(precision=precision)
        # each component equals the single-component inverse of its coefficients
        for a in V.VectorField.CanonicalIndices():
            f = torch.zeros_like(u[a].Data())
            grid.inverse_batch(L, a, e[a].Data(), f, precision)
            assert torch.equal(f, u[a].Data()), a
        back = V.VectorExpansion.of(u, precision)
        for a in V.VectorExpansion.CanonicalIndices():
            assert relerr(back[a].Data().cpu().numpy(), e[a].Data().cpu().numpy()) < tol, a
