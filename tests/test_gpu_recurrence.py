"""FP64 transforms with the Wigner values generated by the l-recurrence inside
the contraction kernels (no stored table).

The recurrence is the table build's (Wigner.h:347-472, exponent-extended
start values), carried for d_k / s_k so that each step is two FMAs. The bar
is the FP64 drop-in tolerance against the golden fixtures, the C restatement
and the reference, plus agreement with the stored-table path of the same
grid: 1e-14 up to lmax 160; at lmax 2048 the two recurrences' own rounding
(the same recursion, rounded differently over 2000 steps) separates the
forward results by ~9e-15, so the bar there is 3e-14, still 5x below the
round-trip error both paths share (1.5e-13).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import golden_cases, relerr

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module")
def gsht():
    import gshtrans_b200

    return gshtrans_b200


def _zero_grid(g, is_real, count=None):
    shape = g.FieldSize() if count is None else (count, g.FieldSize())
    return np.zeros(shape, np.float64 if is_real else np.complex128)


def test_golden_transforms_without_a_table(gsht, golden):
    tr = golden["transforms"]
    grids = {}
    try:
        for i, L, lmax, n, is_real in golden_cases(tr):
            key = (L, max(abs(n), 3))
            if key not in grids:
                grids[key] = gsht.GaussLegendreGrid(L, key[1], forms=("recurrence",))
            g = grids[key]
            c = tr[f"c{i}_coef"]
            f = _zero_grid(g, is_real)
            g.InverseTransformation(lmax, n, c, f)
            if lmax == 0:
                assert f[0] == pytest.approx(tr[f"c{i}_grid"][0], rel=1e-15)
            else:
                assert relerr(f, tr[f"c{i}_grid"]) < TOL, i
            acc = tr[f"c{i}_acc_init"].copy()
            g.ForwardTransformation(lmax, n, tr[f"c{i}_grid"], acc)
            assert relerr(acc, tr[f"c{i}_acc"]) < TOL, i
            if not is_real and lmax == L:
                assert acc[-1] == 0  # c_{L,L} zeroed (GaussLegendreGrid.h:209-215)
    finally:
        for g in grids.values():
            g.close()


@pytest.mark.parametrize("seed", range(4))
def test_random_sizes_vs_restated(gsht, restated, seed):
    # tests/CheckCoeff2Coeff.h:40-84 with seeds, on a grid without a table.
    rng = np.random.default_rng(3000 + seed)
    L = int(rng.integers(4, 257))
    lmax = int(rng.integers(4, L + 1))
    nmax = min(lmax, 4)
    n = int(rng.integers(-nmax, nmax + 1))
    with gsht.GaussLegendreGrid(L, nmax, forms=("recurrence",)) as g:
        for is_real in (False, True):
            c = oracle.random_coefficients(rng, L, lmax, n, is_real)
            f = _zero_grid(g, is_real)
            g.InverseTransformation(lmax, n, c, f)
            assert relerr(f, restated.inverse(L, lmax, n, is_real, c)) < TOL
            out = np.zeros_like(c)
            g.ForwardTransformation(lmax, n, f, out)
            assert relerr(out, restated.forward(L, lmax, n, is_real, f)) < TOL


@pytest.mark.parametrize("count", [1, 2, 3, 9])
def test_batches_match_the_stored_table(gsht, count):
    # count 1..9 complex fields = 2..18 rows: every row-group width of the
    # inverse (1, 2, 4, 8 rows) and forward (1, 2, 4) kernels, with ragged
    # last groups; the same grid holds both forms.
    import torch

    L, n = 160, -2
    rng = np.random.default_rng(40 + count)
    with gsht.GaussLegendreGrid(L, 2, forms=("recurrence",) + ("fp64",)) as g:
        for is_real in (False, True):
            cs = np.stack([oracle.random_coefficients(rng, L, L, n, is_real, 1.0)
                           for _ in range(count)])
            dc = torch.from_numpy(cs).cuda()
            out = {}
            for prec in ("fp64", "recurrence"):
                df = torch.zeros((count, g.FieldSize()),
                                 dtype=torch.float64 if is_real else torch.complex128, device="cuda")
                g.inverse_batch(L, n, dc, df, prec)
                back = torch.zeros_like(dc)
                g.forward_batch(L, n, df, back, prec)
                torch.cuda.synchronize()
                out[prec] = (df.cpu().numpy(), back.cpu().numpy())
            assert relerr(out["recurrence"][0], out["fp64"][0]) < 1e-14
            assert relerr(out["recurrence"][1], out["fp64"][1]) < 1e-14
            assert relerr(out["recurrence"][1], cs) < 1e-12


def test_partial_degree_and_accumulate(gsht, restated):
    # lmax < L: the recurrence stops at lmax; the forward adds into out.
    L, lmax, n = 120, 77, 1
    rng = np.random.default_rng(5)
    with gsht.GaussLegendreGrid(L, 1, nrange=gsht.NonNegative, forms=("recurrence",)) as g:
        c = oracle.random_coefficients(rng, L, lmax, n, False)
        f = _zero_grid(g, False)
        g.InverseTransformation(lmax, n, c, f)
        assert relerr(f, restated.inverse(L, lmax, n, False, c)) < TOL
        acc = c.copy()
        g.ForwardTransformation(lmax, n, f, acc)
        assert relerr(acc, c + restated.forward(L, lmax, n, False, f)) < TOL


def test_L2048_without_a_table_matches_the_stored_table(gsht):
    # The large single-field case: ring lengths 4096, start values that
    # underflow double near the poles (exponent-extended chains).
    import torch

    L, n = 2048, 1
    rng = np.random.default_rng(2048)
    c = torch.from_numpy(oracle.random_coefficients(rng, L, L, n, False, 2.0)).cuda()
    res = {}
    with gsht.GaussLegendreGrid(L, 1, nrange=gsht.Single, forms=("recurrence", "fp64")) as g:
        for prec in ("fp64", "recurrence"):
            f = torch.zeros(g.FieldSize(), dtype=torch.complex128, device="cuda")
            g.InverseTransformation(L, n, c, f, prec)
            back = torch.zeros_like(c)
            g.ForwardTransformation(L, n, f, back, prec)
            torch.cuda.synchronize()
            res[prec] = (f.cpu().numpy(), back.cpu().numpy())
    assert relerr(res["recurrence"][0], res["fp64"][0]) < 3e-14
    assert relerr(res["recurrence"][1], res["fp64"][1]) < 3e-14
    assert relerr(res["recurrence"][1], c.cpu().numpy()) < 1e-12


def test_accuracy_at_least_the_references(gsht, reference):
    # As for the stored table: no further from the reference's long-double
    # instantiation than the reference's double build is.
    L = 384
    rng = np.random.default_rng(385)
    rd = reference.grid(L, 1, 0, 0)
    rl = reference.grid(L, 1, 0, 0, long_double=True)
    try:
        with gsht.GaussLegendreGrid(L, 1, forms=("recurrence",)) as g:
            for is_real, n in ((False, 1), (True, 0)):
                c = oracle.random_coefficients(rng, L, L, n, is_real)
                truth = rl.inverse(L, n, is_real, c)
                f = _zero_grid(g, is_real)
                g.InverseTransformation(L, n, c, f)
                e_gpu, e_ref = relerr(f, truth), relerr(rd.inverse(L, n, is_real, c), truth)
                assert e_gpu <= 1.1 * e_ref + 1e-15, ("inverse", is_real, e_gpu, e_ref)
                truth_c = rl.forward(L, n, is_real, truth)
                out = np.zeros_like(c)
                g.ForwardTransformation(L, n, truth, out)
                e_gpu, e_ref = relerr(out, truth_c), relerr(rd.forward(L, n, is_real, truth), truth_c)
                assert e_gpu <= 1.1 * e_ref + 1e-15, ("forward", is_real, e_gpu, e_ref)
    finally:
        rd.close()
        rl.close()


def test_forms_that_need_a_table_are_refused(gsht):
    with gsht.GaussLegendreGrid(32, 0, forms=("recurrence",)) as g:
        c = oracle.random_coefficients(np.random.default_rng(1), 32, 32, 0, False)
        f = _zero_grid(g, False)
        for prec in ("bf16x3", "ozaki"):
            with pytest.raises(gsht.GSHTError):
                g.InverseTransformation(32, 0, c, f, prec)
        g.InverseTransformation(32, 0, c, f, "recurrence")
    with gsht.GaussLegendreGrid(32, 0) as g:  # table only
        with pytest.raises(gsht.GSHTError):
            g.InverseTransformation(32, 0, c, _zero_grid(g, False), "recurrence")
