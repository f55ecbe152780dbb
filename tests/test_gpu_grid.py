"""GPU grid construction: Gauss-Legendre nodes and the Wigner tables
(GaussLegendreGrid.h:38-73, Wigner.h:24-486) against the oracle."""

from __future__ import annotations

import numpy as np
import pytest
from scipy import special

import oracle
from conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gsht():
    import gshtrans_b200

    return gshtrans_b200


@pytest.mark.parametrize("L", [4, 8, 33, 64, 1024])
def test_nodes_match_reference(gsht, golden, L):
    with gsht.GaussLegendreGrid(L, 0, nrange=gsht.Single) as g:
        th = g.CoLatitudes()
        w = g.CoLatitudeWeights()
    np.testing.assert_allclose(th, golden["nodes"][f"theta_{L}"], rtol=4e-16, atol=0)
    np.testing.assert_allclose(w, golden["nodes"][f"weight_{L}"], rtol=5e-14, atol=0)
    assert abs(w.sum() - 2.0) < 1e-13


def test_wigner_blocks_match_reference_fixture(gsht, golden):
    wig = golden["wigner"]
    grids = {33: gsht.GaussLegendreGrid(33, 3), 64: gsht.GaussLegendreGrid(64, 2)}
    for key in wig.files:
        L = int(key.split("_")[0][1:])
        n = int(key.split("_")[1][1:])
        it = int(key.split("_")[2][1:])
        got = grids[L].Wigner(n, it)
        want = wig[key]
        assert got.shape == want.shape
        # Entry-wise relative to the block's largest value: recurrences with
        # different rounding differ by O(l^2 eps) next to the poles.
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 1e-13, (key, err)
    for g in grids.values():
        g.close()


def test_wigner_nonnegative_orders_layout(gsht):
    # MRange = NonNegative blocks hold m = 0..l only (Indexing.h:118-131).
    with gsht.GaussLegendreGrid(16, 2, mrange=gsht.NonNegative) as gn, \
         gsht.GaussLegendreGrid(16, 2) as ga:
        for n in (-2, 0, 2):
            a = ga.Wigner(n, 5)
            b = gn.Wigner(n, 5)
            ls, ms = oracle.degree_order(16, n, False)
            np.testing.assert_array_equal(b, a[ms >= 0])


def test_wigner_vs_sph_legendre_n0(gsht):
    # tests/CheckLegendre.h criterion (absolute 1e5 eps), at every GL node.
    L = 300
    with gsht.GaussLegendreGrid(L, 0, nrange=gsht.Single) as g:
        th = g.CoLatitudes()
        ls, ms = oracle.degree_order(L, 0, False)
        for it in (0, 7, 150, 299, 300):
            d = g.Wigner(0, it)
            want = special.sph_legendre_p(ls, ms, th[it])[0]
            big = np.abs(want) > 1000 * np.finfo(float).tiny
            assert np.abs(d[big] - want[big]).max() < 1e5 * np.finfo(float).eps


def test_wigner_addition_theorem(gsht):
    # tests/CheckAdditionTheorem.h with the Ortho norm: sum_m d^l_mn d^l_mn'
    # = delta_nn' (2l+1)/(4 pi).
    L = 40
    with gsht.GaussLegendreGrid(L, L) as g:
        for it in (0, 13, 20):
            blocks = {n: g.Wigner(n, it) for n in range(-L, L + 1)}
            for n in (-L, -3, 0, 5, L):
                for npr in (-2, 0, 2, n):
                    for l in range(max(abs(n), abs(npr)), L + 1):
                        a = blocks[n][l * l - n * n:l * l - n * n + 2 * l + 1]
                        b = blocks[npr][l * l - npr * npr:l * l - npr * npr + 2 * l + 1]
                        s = np.dot(a, b) * 4 * np.pi / (2 * l + 1) - (1.0 if n == npr else 0.0)
                        assert abs(s) < 1000 * np.finfo(float).eps


def test_wigner_L1024_vs_restated(gsht, restated):
    L = 1024
    with gsht.GaussLegendreGrid(L, 2, nrange=gsht.Single) as g:
        th = g.CoLatitudes()
        for it in (0, 3, 511, 512, 1021, 1024):
            got = g.Wigner(2, it)
            want = restated.wigner_block(L, 2, th[it])
            assert relerr(got, want) < 1e-12, it


def test_wigner_L2048_unitarity_where_reference_underflows(gsht):
    # The reference's exp(lgamma) start values underflow for L >~ 1930; the
    # exponent-extended start values keep sum_m d^l_{mn}^2 = (2l+1)/(4 pi).
    L = 2048
    with gsht.GaussLegendreGrid(L, 1, nrange=gsht.Single) as g:
        for it in (0, 200, 1024):
            d = g.Wigner(1, it)
            for l in (1, 700, 1500, 2048):
                blk = d[l * l - 1:l * l - 1 + 2 * l + 1]
                s = np.dot(blk, blk) * 4 * np.pi / (2 * l + 1)
                assert abs(s - 1.0) < 1e-11, (it, l, s)


def _block_sizes(lmax, mmax, ns, all_m=True):
    out = []
    for n in ns:
        s = 0
        for l in range(abs(n), lmax + 1):
            t = min(l, mmax)
            s += 2 * t + 1 if all_m else t + 1
        out.append(s)
    return out


def test_wigner_compute_matches_reference_fixture(gsht, golden):
    # Wigner<double, Norm, All, All>(lMax, mMax, nMax, theta), reference values.
    ws = golden["wigner_single"]
    for i in range(int(ws["count"])):
        lmax, mmax, nmax, fp = (int(x) for x in ws[f"c{i}_meta"])
        got = gsht.wigner(lmax, mmax, nmax, ws[f"c{i}_theta"], mrange=gsht.All,
                          nrange=gsht.All, four_pi=bool(fp))
        want = ws[f"c{i}_values"]
        assert got.shape == want.shape, i
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 1e-13, (i, err)


def test_wigner_compute_storage_and_ranges(gsht):
    L, M, N = 20, 7, 3
    th = np.array([0.3, 1.1, 2.5])
    ns = list(range(-N, N + 1))
    sizes = _block_sizes(L, M, ns)
    col = gsht.wigner(L, M, N, th, nrange=gsht.All)
    row = gsht.wigner(L, M, N, th, nrange=gsht.All, row_major=True)
    assert col.size == row.size == 3 * sum(sizes)
    # ColumnMajor: n outer, angle inner; RowMajor: angle outer, n inner.
    blocks_col, off = {}, 0
    for n, sz in zip(ns, sizes):
        for it in range(3):
            blocks_col[(n, it)] = col[off:off + sz]
            off += sz
    off = 0
    for it in range(3):
        for n, sz in zip(ns, sizes):
            np.testing.assert_array_equal(row[off:off + sz], blocks_col[(n, it)])
            off += sz
    # One angle at a time gives the same blocks.
    for it in range(3):
        one = gsht.wigner(L, M, N, th[it], nrange=gsht.All)
        np.testing.assert_array_equal(one, np.concatenate([blocks_col[(n, it)] for n in ns]))
    # NRange NonNegative / Single select blocks; MRange NonNegative keeps m >= 0.
    nn = gsht.wigner(L, M, N, th, nrange=gsht.NonNegative)
    np.testing.assert_array_equal(
        nn, np.concatenate([blocks_col[(n, it)] for n in range(0, N + 1) for it in range(3)]))
    single = gsht.wigner(L, M, N, th, nrange=gsht.Single)
    np.testing.assert_array_equal(single, np.concatenate([blocks_col[(N, it)] for it in range(3)]))
    half = gsht.wigner(L, M, N, th, mrange=gsht.NonNegative, nrange=gsht.All)
    parts = []
    for n in ns:
        for it in range(3):
            b, o = blocks_col[(n, it)], 0
            for l in range(abs(n), L + 1):
                t = min(l, M)
                parts.append(b[o + t:o + 2 * t + 1])
                o += 2 * t + 1
    np.testing.assert_array_equal(half, np.concatenate(parts))


def test_wigner_compute_equals_grid_tables(gsht):
    L = 64
    with gsht.GaussLegendreGrid(L, 2) as g:
        th = g.CoLatitudes()
        first = _block_sizes(L, L, [-2])[0]
        for it in (0, 17, 64):
            cases = {
                2: gsht.wigner(L, L, 2, th[it], nrange=gsht.Single),
                0: gsht.wigner(L, L, 0, th[it], nrange=gsht.Single),
                -2: gsht.wigner(L, L, 2, th[it], nrange=gsht.All)[:first],
            }
            for n, got in cases.items():
                want = g.Wigner(n, it)
                # The grid's -m rows come from the table at the mirrored node
                # (pi - theta symmetry), so they differ in the last bits.
                assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max(), (n, it)
