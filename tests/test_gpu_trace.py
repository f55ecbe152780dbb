"""Per-role cycle trace of the tensor-core Legendre kernels
(gsht_tc_trace_enable / gsht_tc_trace_read): the traced kernel copies give
the same results bit for bit, and their counters are consistent (every
wait inside its role's span, one MMA issuer per CTA or per CTA pair)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _round(g, L, n, c, prec):
    import torch

    dc = torch.from_numpy(c).cuda()
    f = torch.zeros((c.shape[0], g.FieldSize()), dtype=torch.complex128, device="cuda")
    g.inverse_batch(L, n, dc, f, prec)
    back = torch.zeros_like(dc)
    g.forward_batch(L, n, f, back, prec)
    torch.cuda.synchronize()
    g.device_status()
    return f.cpu().numpy(), back.cpu().numpy()


@pytest.mark.parametrize("prec", ["bf16x3", "ozaki"])
def test_traced_kernels_match_and_count_consistently(prec):
    import gshtrans_b200 as gsht

    L, n, B = 192, 1, 64
    rng = np.random.default_rng(7)
    c = np.stack([oracle.random_coefficients(rng, L, L, n, False, 1.5) for _ in range(B)])
    with gsht.GaussLegendreGrid(L, 1, forms=(prec,)) as g:
        plain = _round(g, L, n, c, prec)
        with gsht.TensorCoreTrace() as tr:
            traced = _round(g, L, n, c, prec)
            counters = [tr.read(prec, d) for d in (0, 1)]
    assert np.array_equal(plain[0], traced[0]) and np.array_equal(plain[1], traced[1])
    for d, k in enumerate(counters):
        assert k["ctas"] > 0 and 0 < k["mma_ctas"] <= k["ctas"], (d, k)
        assert 0 <= k["producer_wait_free_stage"] <= k["producer"], (d, k)
        assert 0 <= k["mma_wait_loaded_stage"] + k["mma_wait_epilogue"] <= k["mma"], (d, k)
        assert 0 <= k["epilogue_wait_accumulators"] <= k["epilogue"], (d, k)
        assert 0.0 <= k["mma_frac_issuing"] <= 1.0
    if prec == "bf16x3":
        # 256 field rows: the forward runs in CTA pairs, one issuer per pair
        assert counters[1]["mma_ctas"] * 2 == counters[1]["ctas"]
        assert counters[0]["mma_ctas"] == counters[0]["ctas"]

