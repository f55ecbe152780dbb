"""CPU stand-ins of the four sharded stages (test infrastructure).

They restate, in NumPy on the oracle's Wigner blocks and FFT
(oracle/gsht_oracle.c, following GaussLegendreGrid.h:163-216 and
:281-320), what gsht_forward_rings / gsht_forward_orders /
gsht_inverse_orders / gsht_inverse_rings compute, on CPU torch tensors in
the library's spectra layout [m][sign][field][pitch] (-m rows at the mirrored
colatitude). With them the exchange logic of gshtrans_b200.sharded runs over
gloo on CPU and is compared with the oracle's whole transforms.
"""

from __future__ import annotations

import numpy as np

import oracle


class OracleStages:
    def __init__(self, L, n):
        self.R = oracle.Restated()
        self.L, self.n = L, n
        self.theta, self.w = self.R.nodes(L)
        self.nt, self.nphi = L + 1, 2 * L
        self.pitch = (self.nt + 15) // 16 * 16
        self.blocks = [self.R.wigner_block(L, n, t) for t in self.theta]

    def new_spectra(self, lmax, is_real, count, like):
        import torch

        return torch.zeros((lmax + 1, 1 if is_real else 2, count, self.pitch), dtype=torch.complex128)

    def _d(self, j, l, m):
        # GSHIndices<All>(L, L, n) block: degree offset l^2 - n^2, order m + l
        return self.blocks[j][l * l - self.n * self.n + l + m]

    @staticmethod
    def _idx(l, m, n, is_real):
        na = abs(n)
        if is_real:
            return l * (l + 1) // 2 - na * (na + 1) // 2 + m
        return l * l - n * n + l + m

    def forward_rings(self, lmax, is_real, count, begin, end, grid_values, spectra):
        g = grid_values.numpy().reshape(count, self.nt, self.nphi)
        s = spectra.numpy()
        for f in range(count):
            for j in range(begin, end):
                F = self.R.fft(g[f, j].astype(np.complex128), -1)
                scale = self.w[j] * 2 * np.pi / self.nphi
                for m in range(lmax + 1):
                    s[m, 0, f, j] = F[m] * scale
                    if not is_real:
                        s[m, 1, f, self.nt - 1 - j] = F[self.nphi - m] * scale if m else 0

    def forward_orders(self, lmax, n, is_real, count, begin, end, spectra, coef):
        s = spectra.numpy()
        c = coef.numpy().reshape(count, -1)
        for f in range(count):
            for m in range(begin, end):
                for l in range(max(m, abs(n)), lmax + 1):
                    c[f, self._idx(l, m, n, is_real)] += sum(
                        self._d(j, l, m) * s[m, 0, f, j] for j in range(self.nt))
                    if not is_real and m > 0:
                        c[f, self._idx(l, -m, n, False)] += sum(
                            self._d(j, l, -m) * s[m, 1, f, self.nt - 1 - j] for j in range(self.nt))

    def inverse_orders(self, lmax, n, is_real, count, begin, end, coef, spectra):
        s = spectra.numpy()
        c = coef.numpy().reshape(count, -1)
        for f in range(count):
            for m in range(begin, end):
                for j in range(self.nt):
                    ls = range(max(m, abs(n)), lmax + 1)
                    s[m, 0, f, j] = sum(c[f, self._idx(l, m, n, is_real)] * self._d(j, l, m) for l in ls)
                    if not is_real:
                        s[m, 1, f, self.nt - 1 - j] = (
                            sum(c[f, self._idx(l, -m, n, False)] * self._d(j, l, -m) for l in ls)
                            if m else 0)

    def inverse_rings(self, lmax, is_real, count, begin, end, spectra, grid_values):
        s = spectra.numpy()
        g = grid_values.numpy().reshape(count, self.nt, self.nphi)
        for f in range(count):
            for j in range(begin, end):
                X = np.zeros(self.nphi, np.complex128)
                for m in range(lmax + 1):
                    X[m] += s[m, 0, f, j]
                    if not is_real and m > 0:
                        X[self.nphi - m] += s[m, 1, f, self.nt - 1 - j]
                if is_real:
                    # c2r: Hermitian extension, imaginary parts of bins 0 and N/2 dropped
                    X[0] = X[0].real
                    h = self.nphi // 2
                    X[h] = X[h].real
                    for m in range(1, h):
                        X[self.nphi - m] = np.conj(X[m])
                    g[f, j] = self.R.fft(X, +1).real
                else:
                    g[f, j] = self.R.fft(X, +1)
