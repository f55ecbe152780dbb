"""Generates the golden fixtures in tests/golden from the REFERENCE itself.

The reference GSHTrans headers are compiled in place (oracle/Makefile ->
oracle/_ref/libgsht_ref.so, with the FFTWpp/GaussQuad stand-ins of
oracle/shim) and driven through oracle.Reference. Every fixture stores the
seeded inputs together with the reference's outputs:

  nodes.npz        colatitudes/weights for several grid degrees
  wigner.npz       table blocks d^l_{mn}(theta_j) (GSHIndices<All> layout)
  transforms.npz   inverse / forward / forward-accumulate cases
  wigner_single.npz  Wigner<double, Norm, All, All>(lMax, mMax, nMax, theta)
                     at one angle (tests/CheckAdditionTheorem.h:27 form)
  lmax2048.npz     the large single-transform case (lmax 2048, n = 1) in long
                   double: inverse rings and forward orders (see make_lmax2048)

Run from the repository root:  python tests/golden/make_golden.py
(``--only-lmax2048`` regenerates lmax2048.npz alone; it takes several minutes
of CPU: the long-double table is rebuilt chunk by chunk for the forward)
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

# (grid L, lmax, n, is_real, seed, envelope) — grid degrees chosen to cover
# the FFT lengths 2L = 16 (2^4), 66 (2*3*11), 128 (cfg 1), 20 (4*5), 12, 14
# (2*7), and truncation lmax < L.
CASES = [
    (8, 8, 0, False, 1, None),
    (8, 8, 2, True, 2, None),
    (8, 5, -1, False, 3, None),
    (33, 33, -2, False, 4, 1.0),
    (33, 33, 3, True, 5, 1.0),
    (33, 20, 1, True, 6, None),
    (64, 64, 0, False, 7, 1.0),   # the L = 64 round-trip case: n = 0, envelope 1/(l+1)
    (10, 10, 0, True, 8, None),
    (6, 6, 1, False, 9, None),
    (7, 7, -3, True, 10, None),
    (7, 7, 2, False, 11, None),
    (33, 0, 0, False, 12, None),  # lmax == 0 special case (complex)
    (33, 0, 0, True, 13, None),   # lmax == 0 special case (real)
]


# (lmax, mmax, nmax, theta, fourPi) for wigner_single.npz: mMax == lMax and
# mMax < lMax, both normalisations, angles near a pole and mid-sphere.
WIGNER_SINGLE = [
    (16, 16, 4, 0.7, False),
    (16, 16, 4, 0.7, True),
    (24, 9, 3, 2.9, False),
    (24, 9, 3, 0.05, True),
]


def make_wigner_single(ref):
    ws = {}
    for i, (lmax, mmax, nmax, theta, four_pi) in enumerate(WIGNER_SINGLE):
        ws[f"c{i}_meta"] = np.array([lmax, mmax, nmax, int(four_pi)])
        ws[f"c{i}_theta"] = np.array([theta])
        ws[f"c{i}_values"] = ref.wigner_single(lmax, mmax, nmax, theta, four_pi=four_pi)
    ws["count"] = np.array(len(WIGNER_SINGLE))
    np.savez_compressed(os.path.join(HERE, "wigner_single.npz"), **ws)


# The large single-transform case: lmax 2048 (nTheta 2049, nPhi 4096),
# upper index n = 1, coefficients with envelope (l+1)^-2. The reference's
# double build cannot serve there (its start values underflow and its table
# does not fit in host memory), so the reference's Wigner is instantiated in
# long double on chunks of colatitudes (oracle.Reference.chunked_*). Stored:
# the inverse on the rings below (both poles, the region near theta 0.37
# where the double start values underflow, the equator) and the forward of a
# seeded white-noise grid on the orders below. The inputs are regenerated in
# the tests from their seeds; checksums of them are stored to catch drift.
LMAX2048 = 2048
N2048 = 1
RINGS2048 = [0, 1, 2, 5, 30, 120, 240, 241, 480, 1024, 1500, 1808, 2030, 2046, 2047, 2048]
ORDERS2048_COMPLEX = [-2048, -2047, -1700, -1024, -300, -2, -1, 0, 1, 2, 3, 240, 1023, 1800,
                      2046, 2047, 2048]
ORDERS2048_REAL = [0, 1, 2, 240, 1023, 1800, 2047, 2048]
SEEDS2048 = {False: (2048, 4096), True: (2049, 4097)}  # (coefficients, grid) per is_real


def lmax2048_inputs(is_real):
    """Seeded coefficients (envelope (l+1)^-2) and white-noise grid of the
    lmax 2048 fixture."""
    L, n = LMAX2048, N2048
    cs, gs = SEEDS2048[is_real]
    c = oracle.random_coefficients(np.random.default_rng(cs), L, L, n, is_real, 2.0)
    rng = np.random.default_rng(gs)
    shape = (L + 1, 2 * L)
    grid = rng.standard_normal(shape)
    if not is_real:
        grid = grid + 1j * rng.standard_normal(shape)
    return c, grid


def make_lmax2048(ref):
    import time

    L, n = LMAX2048, N2048
    out = {"meta": np.array([L, n]), "rings": np.array(RINGS2048)}
    th, w = ref.chunked_nodes(L)
    out["theta"], out["weight"] = th, w
    for is_real in (False, True):
        k = "real" if is_real else "complex"
        orders = ORDERS2048_REAL if is_real else ORDERS2048_COMPLEX
        c, grid = lmax2048_inputs(is_real)
        out[f"{k}_coef_sum"] = np.array(c.sum())
        out[f"{k}_coef_head"] = np.concatenate([c[:8], c[-8:]])
        out[f"{k}_grid_sum"] = np.array(grid.sum())
        out[f"{k}_orders"] = np.array(orders)
        t0 = time.time()
        inv = ref.chunked_inverse_rings(L, n, is_real, c, RINGS2048)
        inv64 = ref.chunked_inverse_rings(L, n, is_real, c, RINGS2048, long_double=False)
        t1 = time.time()
        fwd = ref.chunked_forward_orders(L, n, is_real, grid, orders)
        fwd64 = ref.chunked_forward_orders(L, n, is_real, grid, orders, long_double=False)
        t2 = time.time()
        out[f"{k}_inverse_rings"] = inv
        ld = np.concatenate([fwd[m] for m in orders])
        out[f"{k}_forward_orders"] = ld
        # the reference's own double build on the same inputs, as an error figure
        d64 = np.concatenate([fwd64[m] for m in orders])
        out[f"{k}_ref64_inverse_relerr"] = np.array(np.linalg.norm(inv64 - inv) / np.linalg.norm(inv))
        out[f"{k}_ref64_forward_relerr"] = np.array(np.linalg.norm(d64 - ld) / np.linalg.norm(ld))
        print(k, "inverse %.1f s, forward %.1f s" % (t1 - t0, t2 - t1),
              "reference double vs long double: inverse %.2e forward %.2e"
              % (out[f"{k}_ref64_inverse_relerr"], out[f"{k}_ref64_forward_relerr"]))
    np.savez_compressed(os.path.join(HERE, "lmax2048.npz"), **out)


def main():
    ref = oracle.Reference()
    if "--only-wigner-single" in sys.argv:
        make_wigner_single(ref)
        return
    if "--only-lmax2048" in sys.argv:
        make_lmax2048(ref)
        return
    make_wigner_single(ref)
    make_lmax2048(ref)
    nodes = {}
    for L in (4, 8, 33, 64, 1024):
        g = ref.grid(L, 0, 0, 2)
        th, w = g.nodes()
        nodes[f"theta_{L}"] = th
        nodes[f"weight_{L}"] = w
        g.close()
    np.savez_compressed(os.path.join(HERE, "nodes.npz"), **nodes)

    wig = {}
    g = ref.grid(33, 3, 0, 0)
    for n in range(-3, 4):
        for it in (0, 1, 16, 32, 33):
            wig[f"L33_n{n}_t{it}"] = g.wigner_block(n, it)
    g.close()
    g = ref.grid(64, 2, 0, 0)
    for n in (-2, 0, 2):
        for it in (0, 32, 64):
            wig[f"L64_n{n}_t{it}"] = g.wigner_block(n, it)
    g.close()
    np.savez_compressed(os.path.join(HERE, "wigner.npz"), **wig)

    tr = {}
    grids = {}
    for i, (L, lmax, n, is_real, seed, env) in enumerate(CASES):
        key = (L, max(abs(n), 3))
        if key not in grids:
            grids[key] = ref.grid(L, key[1], 0, 0)
        g = grids[key]
        rng = np.random.default_rng(seed)
        c = oracle.random_coefficients(rng, L, lmax, n, is_real, env)
        f = g.inverse(lmax, n, is_real, c)
        fwd = g.forward(lmax, n, is_real, f)
        init = rng.standard_normal(c.size) + 1j * rng.standard_normal(c.size)
        acc = g.forward(lmax, n, is_real, f, out=init.copy())
        p = f"c{i}_"
        tr[p + "meta"] = np.array([L, lmax, n, int(is_real)])
        tr[p + "coef"] = c
        tr[p + "grid"] = f
        tr[p + "fwd"] = fwd
        tr[p + "acc_init"] = init
        tr[p + "acc"] = acc
    for g in grids.values():
        g.close()
    tr["count"] = np.array(len(CASES))
    np.savez_compressed(os.path.join(HERE, "transforms.npz"), **tr)
    for name in ("nodes.npz", "wigner.npz", "transforms.npz", "wigner_single.npz", "lmax2048.npz"):
        print(name, os.path.getsize(os.path.join(HERE, name)))


if __name__ == "__main__":
    main()
