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

Run from the repository root:  python tests/golden/make_golden.py
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


def main():
    ref = oracle.Reference()
    if "--only-wigner-single" in sys.argv:
        make_wigner_single(ref)
        return
    make_wigner_single(ref)
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
    for name in ("nodes.npz", "wigner.npz", "transforms.npz", "wigner_single.npz"):
        print(name, os.path.getsize(os.path.join(HERE, name)))


if __name__ == "__main__":
    main()
