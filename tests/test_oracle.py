"""Pins the CPU oracle (oracle/gsht_oracle.c) against the reference.

The golden fixtures were produced by the reference headers themselves
(tests/golden/make_golden.py). Where the reference build oracle/_ref exists
the restatement is also compared with it on fresh seeded inputs, and the
reference's own test properties (tests/CheckLegendre.h,
tests/CheckAdditionTheorem.h, tests/CheckCoeff2Coeff.h) are re-run.
"""

from __future__ import annotations

import numpy as np
import pytest
from scipy import special

import oracle
from conftest import golden_cases, relerr


def test_restated_nodes_match_reference_fixture(golden, restated):
    for L in (4, 8, 33, 64, 1024):
        th, w = restated.nodes(L)
        np.testing.assert_array_equal(th, golden["nodes"][f"theta_{L}"])
        np.testing.assert_array_equal(w, golden["nodes"][f"weight_{L}"])


def test_restated_wigner_bit_exact_vs_reference_fixture(golden, restated):
    wig = golden["wigner"]
    nodes = golden["nodes"]
    for key in wig.files:
        L = int(key.split("_")[0][1:])
        n = int(key.split("_")[1][1:])
        it = int(key.split("_")[2][1:])
        th = nodes[f"theta_{L}"][it]
        got = restated.wigner_block(L, n, th)
        np.testing.assert_array_equal(got, wig[key], err_msg=key)


def test_restated_transforms_vs_reference_fixture(golden, restated):
    tr = golden["transforms"]
    for i, L, lmax, n, is_real in golden_cases(tr):
        c = tr[f"c{i}_coef"]
        f = restated.inverse(L, lmax, n, is_real, c)
        if lmax == 0:
            # Only out[0] is defined by the reference for lmax == 0.
            assert f.ravel()[0] == pytest.approx(tr[f"c{i}_grid"].ravel()[0], rel=1e-15)
        else:
            assert relerr(f, tr[f"c{i}_grid"]) < 1e-14, i
        g = restated.forward(L, lmax, n, is_real, tr[f"c{i}_grid"])
        assert relerr(g, tr[f"c{i}_fwd"]) < 1e-14, i
        acc = restated.forward(L, lmax, n, is_real, tr[f"c{i}_grid"], out=tr[f"c{i}_acc_init"].copy())
        assert relerr(acc, tr[f"c{i}_acc"]) < 1e-14, i


def test_restated_fft_conventions(restated):
    rng = np.random.default_rng(0)
    for N in (1, 2, 6, 12, 66, 128, 502):
        x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
        np.testing.assert_allclose(restated.fft(x, -1), np.fft.fft(x), atol=1e-12 * N)
        np.testing.assert_allclose(restated.fft(x, +1), np.fft.ifft(x) * N, atol=1e-12 * N)


def test_fixture_semantics_of_random_coefficients():
    # GridBase.h:124-172: c_{L,L} = 0 for complex fields at lmax == L; real
    # fields have Im c_{l,0} = 0 and Im c_{L,L} = 0.
    rng = np.random.default_rng(1)
    c = oracle.random_coefficients(rng, 9, 9, 2, False)
    assert c[-1] == 0 and c.size == oracle.size_all(9, 2)
    r = oracle.random_coefficients(rng, 9, 9, -2, True)
    ls, ms = oracle.degree_order(9, -2, True)
    assert np.all(r[ms == 0].imag == 0) and r[-1].imag == 0
    assert r.size == oracle.size_nonneg(9, -2)


# --- the reference itself (where oracle/_ref was built) ---------------------

def test_reference_reproduces_fixture(golden, reference):
    tr = golden["transforms"]
    for i, L, lmax, n, is_real in list(golden_cases(tr))[:4]:
        g = reference.grid(L, max(abs(n), 3), 0, 0)
        f = g.inverse(lmax, n, is_real, tr[f"c{i}_coef"])
        np.testing.assert_array_equal(f, tr[f"c{i}_grid"])
        g.close()


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_restated_matches_reference_random(reference, restated, seed):
    # tests/CheckCoeff2Coeff.h draws lMaxGrid in [4, 256], lMax in [4, lMaxGrid],
    # nMax = min(lMax, 4) and n in [-nMax, nMax]; seeded here.
    rng = np.random.default_rng(100 + seed)
    L = int(rng.integers(4, 97))
    lmax = int(rng.integers(4, L + 1))
    nmax = min(lmax, 4)
    n = int(rng.integers(-nmax, nmax + 1))
    g = reference.grid(L, nmax, 0, 0)
    for is_real in (False, True):
        c = oracle.random_coefficients(rng, L, lmax, n, is_real)
        f_ref = g.inverse(lmax, n, is_real, c)
        f_orc = restated.inverse(L, lmax, n, is_real, c)
        assert relerr(f_orc, f_ref) < 1e-14
        c_ref = g.forward(lmax, n, is_real, f_ref)
        c_orc = restated.forward(L, lmax, n, is_real, f_ref)
        assert relerr(c_orc, c_ref) < 1e-14
        # Round trip, tests/CheckCoeff2Coeff.h:80-83 (50000 eps absolute).
        assert np.max(np.abs(c_ref - c)) < 50000 * np.finfo(float).eps
    g.close()


def test_reference_check_legendre(reference):
    # tests/CheckLegendre.h: n = 0, L = 300, one angle, vs sph_legendre.
    L, theta = 300, 1.234
    d = reference.wigner_single(L, L, 0, theta)
    ls, ms = oracle.degree_order(L, 0, False)
    # std::sph_legendre(l, m, theta) = Y_l^m(theta, 0), the same function as
    # scipy's sph_legendre_p (first row: no derivative).
    want = special.sph_legendre_p(ls, ms, theta)[0]
    # CheckLegendre.h:36-37 divides by `norm = |plmSTD| > tiny`, a bool, so
    # the bound is absolute: |d - sph_legendre| <= 1e5 eps where |value| > tiny.
    big = np.abs(want) > 1000 * np.finfo(float).tiny
    assert np.abs(d[big] - want[big]).max() < 1e5 * np.finfo(float).eps


def test_reference_addition_theorem(reference):
    # tests/CheckAdditionTheorem.h: FourPi norm, L = 40, all n, n'.
    L = 40
    d = reference.wigner_single(L, L, L, 0.7, four_pi=True)
    blocks = {}
    off = 0
    for n in range(-L, L + 1):
        sz = oracle.size_all(L, n)
        blocks[n] = d[off:off + sz]
        off += sz
    for n in (-L, -3, 0, 5, L):
        for npr in (-2, 0, 2, n):
            lmin = max(abs(n), abs(npr))
            for l in range(lmin, L + 1):
                a = blocks[n][l * l - n * n:l * l - n * n + 2 * l + 1]
                b = blocks[npr][l * l - npr * npr:l * l - npr * npr + 2 * l + 1]
                s = np.dot(a, b) - (1.0 if n == npr else 0.0)
                assert abs(s) < 1000 * np.finfo(float).eps


def test_restated_wigner_vs_reference_single_angle_fixture(golden, restated):
    # Wigner<double, Ortho, All, All>(16, 16, 4, 0.7): blocks n = -4..4.
    ws = golden["wigner_single"]
    lmax, mmax, nmax, fp = (int(x) for x in ws["c0_meta"])
    assert (lmax, mmax, fp) == (16, 16, 0)
    th = float(ws["c0_theta"][0])
    got = np.concatenate([restated.wigner_block(lmax, n, th) for n in range(-nmax, nmax + 1)])
    np.testing.assert_array_equal(got, ws["c0_values"])


def test_package_coefficient_generator_matches_the_oracle():
    # bench.py draws its inputs with the package's generator; the tests use
    # the oracle's. Same seed, same arrays.
    import gshtrans_b200 as g

    for L, lmax, n, is_real, env in ((8, 8, 0, False, None), (33, 20, -2, False, 1.0),
                                     (33, 33, 3, True, 1.5), (64, 64, 1, True, None)):
        a = g.random_coefficients(np.random.default_rng(5), L, lmax, n, is_real, env)
        b = oracle.random_coefficients(np.random.default_rng(5), L, lmax, n, is_real, env)
        np.testing.assert_array_equal(a, b)
        la, ma = g.degree_order(lmax, n, is_real)
        lb, mb = oracle.degree_order(lmax, n, is_real)
        np.testing.assert_array_equal(la, lb)
        np.testing.assert_array_equal(ma, mb)


@pytest.mark.parametrize("long_double", [True, False])
def test_chunked_reference_equals_the_whole_grid(reference, long_double):
    # The chunked transforms (the reference's Wigner built on chunks of
    # colatitudes, the loops of GaussLegendreGrid.h:163-216 / 281-320 per
    # chunk) reproduce a whole GaussLegendreGrid<Real, All, Single> bit for bit.
    for L, n in ((40, 1), (33, 2), (64, 0)):
        g = reference.grid(L, n, 0, 2, long_double=long_double)
        try:
            rng = np.random.default_rng(L + n)
            for is_real in (False, True):
                c = oracle.random_coefficients(rng, L, L, n, is_real, 2.0)
                full = g.inverse(L, n, is_real, c).reshape(L + 1, 2 * L)
                rings = [0, 1, L // 2, L - 1, L]
                part = reference.chunked_inverse_rings(L, n, is_real, c, rings, long_double=long_double)
                np.testing.assert_array_equal(part, full[rings])
                grid = rng.standard_normal(full.shape)
                if not is_real:
                    grid = grid + 1j * rng.standard_normal(full.shape)
                whole = g.forward(L, n, is_real, grid.ravel())
                _, ms = oracle.degree_order(L, n, is_real)
                orders = [0, 1, 2, L] + ([] if is_real else [-1, -(L - 1), -L])
                got = reference.chunked_forward_orders(L, n, is_real, grid, orders, chunk=5,
                                                       long_double=long_double)
                for m in orders:
                    np.testing.assert_array_equal(got[m], whole[ms == m])
            th, w = g.nodes()
            th2, w2 = reference.chunked_nodes(L, long_double)
            np.testing.assert_array_equal(th, th2)
            np.testing.assert_array_equal(w, w2)
        finally:
            g.close()


def test_lmax2048_fixture_is_consistent(golden):
    # The seeded inputs regenerate to the stored checksums, the nodes are the
    # mirrored Gauss-Legendre colatitudes, and the reference's own double
    # build misses the long-double values by far more than 1e-12 at this
    # degree (its start values underflow, Wigner.h:77-79).
    import importlib.util
    import os

    from conftest import GOLDEN

    fx = np.load(os.path.join(GOLDEN, "lmax2048.npz"))
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    L, n = (int(v) for v in fx["meta"])
    assert (L, n) == (2048, 1)
    th = fx["theta"]
    assert np.all(np.diff(th) > 0) and np.max(np.abs(th + th[::-1] - np.pi)) < 1e-14
    assert abs(fx["weight"].sum() - 2.0) < 1e-13
    for is_real in (False, True):
        k = "real" if is_real else "complex"
        c, grid = mg.lmax2048_inputs(is_real)
        np.testing.assert_array_equal(np.concatenate([c[:8], c[-8:]]), fx[f"{k}_coef_head"])
        assert abs(c.sum() - fx[f"{k}_coef_sum"][()]) <= 1e-9 * abs(fx[f"{k}_coef_sum"][()])
        assert abs(grid.sum() - fx[f"{k}_grid_sum"][()]) <= 1e-9 * abs(fx[f"{k}_grid_sum"][()])
        assert fx[f"{k}_inverse_rings"].shape == (16, 2 * L)
        assert float(fx[f"{k}_ref64_inverse_relerr"]) > 1e-8
