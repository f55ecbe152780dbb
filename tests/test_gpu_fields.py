"""Fused field expressions (CanonicalComponentField algebra) and the
field-product pipeline (64 pairs at lmax 768) on the GPU.

The pointwise kernel is compared with the same expression evaluated
elementwise in PyTorch (bit-identical for + - * conj real imag; division
within 4 ulps); the pipeline (inverse u, v -> u*v + conj(u)*u -> forward) is
compared with the oracle for one pair and across precision forms.
"""

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


def _rand(grid, count, is_real, seed):
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    shape = (count, grid.FieldSize()) if count > 1 else (grid.FieldSize(),)
    if is_real:
        return torch.randn(shape, generator=g, device="cuda", dtype=torch.float64)
    return torch.complex(torch.randn(shape, generator=g, device="cuda", dtype=torch.float64),
                         torch.randn(shape, generator=g, device="cuda", dtype=torch.float64))


def test_expressions_match_elementwise_reference(gsht):
    import torch

    from gshtrans_b200 import fields as F

    with gsht.GaussLegendreGrid(40, 2) as grid:
        for count in (1, 3):
            a, b, c = (_rand(grid, count, False, s) for s in (1, 2, 3))
            r = _rand(grid, count, True, 4)
            u = F.Field(grid, 1, False, count, a)
            v = F.Field(grid, -1, False, count, b)
            w = F.Field(grid, 0, False, count, c)
            x = F.Field(grid, 0, True, count, r)
            cases = [
                (u * v + F.conj(w) * w, a * b + c.conj() * c),
                (u * v - w * 2.5, a * b - c * 2.5),
                ((u * v) / (w + 1.0), (a * b) / (c + 1.0)),
                (-w + 3.0, -c + 3.0),
                (F.real(u) * x, a.real * r),
                (F.imag(w) + x * x, c.imag + r * r),
            ]
            for expr, want in cases:
                got = expr.evaluate(upper_index=expr.N)
                d = got.Data()
                if want.is_complex() and not d.is_complex():
                    want = want.real
                err = (d - want).abs().max().item() / max(want.abs().max().item(), 1e-300)
                assert err < 4 * np.finfo(float).eps, err
        # reference typing rules: conj keeps N, so u*v + conj(u)*u mixes N=0
        # and N=2 unless the conjugate's index is given
        with pytest.raises(gsht.BadArgument):
            _ = u * v + F.conj(u) * u
        assert (u * v + F.conj(u, upper_index=-1) * u).N == 0
        with pytest.raises(gsht.BadArgument):
            _ = F.Field(grid, 1, False) + F.Field(grid, 0, False)
        with pytest.raises(gsht.BadArgument):
            _ = F.Field(grid, 1, False) / F.Field(grid, 1, False)
        with pytest.raises(gsht.BadArgument):
            _ = F.Field(grid, 1, False) + 1.0


def test_compiled_programs_match_the_interpreter(gsht, monkeypatch):
    """Each program is compiled (NVRTC) into a kernel of its own on first use;
    GSHT_FIELD_JIT=0 runs the interpreting kernel instead. Same arithmetic:
    the two agree to within an ulp or two, and nothing failed to compile."""
    from gshtrans_b200 import fields as F

    with gsht.GaussLegendreGrid(40, 2) as grid:
        a, b, c = (_rand(grid, 3, False, s) for s in (11, 12, 13))
        r = _rand(grid, 3, True, 14)
        u = F.Field(grid, 1, False, 3, a)
        v = F.Field(grid, -1, False, 3, b)
        w = F.Field(grid, 0, False, 3, c)
        x = F.Field(grid, 0, True, 3, r)
        exprs = [u * v + F.conj(w) * w, (u * v) / (w + 1.0) - 0.25, F.real(w) * x + x,
                 -F.imag(w) * 3.0 + x * x, (w * w * w - 1.0) / (w + 2.0)]
        compiled, failed0 = F.jit_stats()
        got = [e.evaluate(upper_index=e.N).Data().clone() for e in exprs]
        compiled1, failed1 = F.jit_stats()
        assert failed1 == failed0 and compiled1 > compiled
        monkeypatch.setenv("GSHT_FIELD_JIT", "0")
        ref = [e.evaluate(upper_index=e.N).Data().clone() for e in exprs]
        for g_, r_ in zip(got, ref):
            err = (g_ - r_).abs().max().item() / max(r_.abs().max().item(), 1e-300)
            assert err < 2 * np.finfo(float).eps, err


def test_compound_assignment_in_place(gsht):
    from gshtrans_b200 import fields as F

    with gsht.GaussLegendreGrid(16, 0) as grid:
        a = _rand(grid, 1, False, 7)
        b = _rand(grid, 1, False, 8)
        u = F.Field(grid, 0, False, 1, a.clone())
        v = F.Field(grid, 0, False, 1, b)
        u += v
        u *= 2.0
        want = (a + b) * 2.0
        assert (u.Data() - want).abs().max().item() < 1e-14


@pytest.mark.parametrize("precision,tol", [("fp64", None), ("bf16x3", 3e-6), ("ozaki", 1e-12)])
def test_field_product_pipeline(gsht, precision, tol):
    # The field-product workload: pairs (u: n=+1, v: n=-1) at lmax 768 (nPhi = 1536 = 2^9 3),
    # envelope (l+1)^-1.5; inverse both, w = u*v + conj(u)*u (upper index 0),
    # forward w at lmax 768. Batched (8 pairs here; the shapes of 64).
    import torch

    from gshtrans_b200 import fields as F

    L, B = 768, 8
    rng = np.random.default_rng(55)
    cu = np.stack([oracle.random_coefficients(rng, L, L, 1, False, 1.5) for _ in range(B)])
    cv = np.stack([oracle.random_coefficients(rng, L, L, -1, False, 1.5) for _ in range(B)])
    forms = () if precision == "fp64" else (precision,)

    def run(prec):
        with gsht.GaussLegendreGrid(L, 1, forms=forms) as grid:
            u = F.Field(grid, 1, False, B)
            v = F.Field(grid, -1, False, B)
            grid.inverse_batch(L, 1, torch.from_numpy(cu).cuda(), u.Data(), prec)
            grid.inverse_batch(L, -1, torch.from_numpy(cv).cuda(), v.Data(), prec)
            w = (u * v + F.conj(u, upper_index=-1) * u).evaluate()
            out = torch.zeros((B, gsht.coefficient_size(L, 0, False)), dtype=torch.complex128, device="cuda")
            grid.forward_batch(L, 0, w.Data(), out, prec)
            grid.device_status()
            return u.Data().cpu().numpy(), w.Data().cpu().numpy(), out.cpu().numpy()

    u64, w64, c64 = run("fp64")
    if precision == "fp64":
        # oracle for the first pair: restated inverse, pointwise product, forward
        R = oracle.Restated()
        fu = R.inverse(L, L, 1, False, cu[0])
        fv = R.inverse(L, L, -1, False, cv[0])
        assert relerr(u64[0], fu) < 1e-13
        fw = fu * fv + np.conj(fu) * fu
        assert relerr(w64[0], fw) < 1e-13
        c_ref = R.forward(L, L, 0, False, fw)
        assert relerr(c64[0], c_ref) < 1e-13
    else:
        _, w_p, c_p = run(precision)
        assert relerr(w_p, w64) < tol
        assert relerr(c_p, c64) < tol
