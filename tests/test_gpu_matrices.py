"""Matrix fields and real vector fields (the reference's header-disabled
MatrixFieldOld / VectorField layers) on the GPU: every pointwise operation
against the same formula written out in NumPy, the conversions between the
real and canonical bases, and transforms of the components."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu

TOL = 1e-14
IDX = (-1, 0, 1)


@pytest.fixture(scope="module")
def gsht():
    import gshtrans_b200

    return gshtrans_b200


def _rand_matrix(M, rng):
    import torch

    d = rng.standard_normal(M.Data().shape) + 1j * rng.standard_normal(M.Data().shape)
    M.Data().copy_(torch.from_numpy(d))
    return {(a, b): d[3 * (a + 1) + (b + 1)] for a in IDX for b in IDX}


def _rand_vector(u, rng):
    import torch

    shape = u.Data().shape
    d = rng.standard_normal(shape)
    if u.Data().is_complex():
        d = d + 1j * rng.standard_normal(shape)
    u.Data().copy_(torch.from_numpy(d))
    return {a: d[a + 1] for a in IDX}


def _np(field):
    return field.Data().cpu().numpy()


def test_matrix_algebra_matches_the_formulas(gsht):
    from gshtrans_b200 import matrices as Mx
    from gshtrans_b200 import vectors as V

    rng = np.random.default_rng(9)
    with gsht.GaussLegendreGrid(12, 2) as g:
        A, B = Mx.MatrixField(g, 2), Mx.MatrixField(g, 2)
        a, b = _rand_matrix(A, rng), _rand_matrix(B, rng)
        u = V.VectorField(g, 2)
        uu = _rand_vector(u, rng)
        # action and product with the canonical metric (MatrixFieldExpressions.h:431-436, 509-513)
        Au = Mx.Action(A, u)
        for al in IDX:
            want = -a[al, -1] * uu[1] + a[al, 0] * uu[0] - a[al, 1] * uu[-1]
            assert relerr(_np(Au[al]), want) < TOL
            assert Au[al].UpperIndex() == al
        AB = Mx.Multiply(A, B)
        for al in IDX:
            for be in IDX:
                want = -a[al, 1] * b[-1, be] + a[al, 0] * b[0, be] - a[al, -1] * b[1, be]
                assert relerr(_np(AB[al, be]), want) < TOL
                assert AB[al, be].UpperIndex() == al + be
        tr = Mx.Trace(A)
        assert relerr(_np(tr), -a[-1, 1] + a[0, 0] - a[1, -1]) < TOL
        det = Mx.Determinant(A)
        want = (-a[-1, -1] * (a[0, 0] * a[1, 1] - a[0, 1] * a[1, 0])
                + a[-1, 0] * (a[0, -1] * a[1, 1] - a[0, 1] * a[1, -1])
                - a[-1, 1] * (a[0, -1] * a[1, 0] - a[0, 0] * a[1, -1]))
        assert relerr(_np(det), want) < TOL
        T, H = Mx.Transpose(A), Mx.Adjoint(A)
        for al in IDX:
            for be in IDX:
                assert np.array_equal(_np(T[al, be]), a[be, al])
                assert np.array_equal(_np(H[al, be]), np.conj(a[be, al]))
        S = A + B - (-A) * 2.0
        for al in IDX:
            for be in IDX:
                assert relerr(_np(S[al, be]), a[al, be] + b[al, be] + 2.0 * a[al, be]) < TOL
        I3 = Mx.Isotropic(g, 1.5 - 0.5j, count=2)
        for al in IDX:
            for be in IDX:
                want = (-1) ** abs(al) * (1.5 - 0.5j) if al + be == 0 else 0.0
                assert np.allclose(_np(I3[al, be]), want, rtol=0, atol=0)
        # the isotropic unit acts as the identity: (g A) u with g = I gives u
        Iu = Mx.Action(Mx.Isotropic(g, 1.0, count=2), u)
        for al in IDX:
            assert relerr(_np(Iu[al]), uu[al]) < TOL


def test_real_vector_conversions(gsht):
    from gshtrans_b200 import vectors as V

    rng = np.random.default_rng(10)
    with gsht.GaussLegendreGrid(10, 1) as g:
        r = V.RealVectorField(g, 3)
        rr = _rand_vector(r, rng)
        c = V.complexify(r)
        assert np.array_equal(_np(c[0]), rr[0] + 0j)
        for al in (-1, 1):
            assert relerr(_np(c[al]), al * rr[1] + 1j * rr[-1]) < TOL
        # canonical components of a real field: c_{-alpha} = (-1)^alpha conj(c_alpha)
        assert relerr(_np(c[-1]), -np.conj(_np(c[1]))) < TOL
        back = V.realify(c)
        for al in IDX:
            assert relerr(_np(back[al]), rr[al]) < TOL
        ip = V.RealInnerProduct(r, back)
        assert relerr(_np(ip), sum(rr[al] * rr[al] for al in IDX)) < TOL
        s = (r + r) * 0.5 - r
        assert np.allclose(_np(s[0]), 0.0, atol=1e-15)


def test_matrix_expansion_round_trip(gsht):
    import torch

    from gshtrans_b200 import matrices as Mx

    L = 24
    rng = np.random.default_rng(11)
    with gsht.GaussLegendreGrid(L, 2) as g:
        E = Mx.MatrixExpansion(g, count=2)
        want = {}
        for al in IDX:
            for be in IDX:
                n = al + be
                c = np.stack([oracle.random_coefficients(rng, L, L, n, False, 1.0) for _ in range(2)])
                E[al, be].Data().copy_(torch.from_numpy(c).view(E[al, be].Data().shape))
                want[al, be] = c
        A = E.to_field()
        E2 = Mx.MatrixExpansion.of(A)
        for al in IDX:
            for be in IDX:
                got = E2[al, be].Data().cpu().numpy().reshape(want[al, be].shape)
                assert relerr(got, want[al, be]) < 1e-13, (al, be)
