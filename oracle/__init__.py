"""CPU oracle for the Gauss-Legendre GSHT path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only to check results against. The product
(``gshtrans_b200`` and ``libgsht_cuda.so``) never imports, links or runs it.

Two oracles live here:

* ``Restated`` — ``gsht_oracle.c``, a plain-C restatement of the reference's
  algorithm (GaussLegendreGrid.h:108-321, Wigner.h:24-486; FFTW's and
  GaussQuad's published algorithms for the two unpinned dependencies).
* ``Reference`` — the unmodified reference headers compiled in place into
  ``_ref/libgsht_ref.so`` (see ``ref_harness.cpp``), available wherever that
  library was built.

Both are pinned against ``tests/golden`` fixtures that the reference build
generated (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
RESTATED_PATH = os.path.join(_HERE, "_build", "liborc.so")
REFERENCE_PATH = os.path.join(_HERE, "_ref", "libgsht_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def size_all(lmax: int, n: int) -> int:
    """GSHIndices<All>(lmax, lmax, n).Size() (Indexing.h:148-150, 104-116)."""
    return (lmax + 1) ** 2 - n * n


def size_nonneg(lmax: int, n: int) -> int:
    """GSHIndices<NonNegative>(lmax, lmax, n).Size() (Indexing.h:118-131)."""
    a = abs(n)
    return (lmax + 1) * (lmax + 2) // 2 - a * (a + 1) // 2


def coef_size(lmax: int, n: int, is_real: bool) -> int:
    return size_nonneg(lmax, n) if is_real else size_all(lmax, n)


def build_restated() -> str:
    if not os.path.exists(RESTATED_PATH) or os.path.getmtime(
        RESTATED_PATH
    ) < os.path.getmtime(os.path.join(_HERE, "gsht_oracle.c")):
        os.system(f"make -s -C {_HERE} restated")
    return RESTATED_PATH


class Restated:
    """ctypes view of the C restatement (gsht_oracle.c)."""

    def __init__(self):
        self.lib = ctypes.CDLL(build_restated())
        L = self.lib
        L.orc_gl_nodes.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_wigner_block.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]
        L.orc_fft.argtypes = [ctypes.c_int, ctypes.c_int, _dp]
        L.orc_fft.restype = None
        for f in (L.orc_forward, L.orc_inverse):
            f.argtypes = [ctypes.c_int] * 4 + [_dp, _dp]

    def nodes(self, L: int):
        th = np.zeros(L + 1)
        w = np.zeros(L + 1)
        assert self.lib.orc_gl_nodes(L + 1, _ptr(th), _ptr(w)) == 0
        return th, w

    def wigner_block(self, L: int, n: int, theta: float) -> np.ndarray:
        out = np.zeros(size_all(L, n))
        assert self.lib.orc_wigner_block(L, n, theta, _ptr(out)) == 0
        return out

    def fft(self, x: np.ndarray, sign: int) -> np.ndarray:
        buf = np.ascontiguousarray(x, dtype=np.complex128).view(np.float64).copy()
        self.lib.orc_fft(len(x), sign, _ptr(buf))
        return buf.view(np.complex128)

    def forward(self, L, lmax, n, is_real, grid, out=None):
        g = np.ascontiguousarray(grid, dtype=np.float64 if is_real else np.complex128)
        if out is None:
            out = np.zeros(coef_size(lmax, n, is_real), np.complex128)
        ob = out.view(np.float64)
        rc = self.lib.orc_forward(L, lmax, n, int(is_real), _ptr(g.view(np.float64)), _ptr(ob))
        assert rc == 0
        return out

    def inverse(self, L, lmax, n, is_real, coef):
        c = np.ascontiguousarray(coef, dtype=np.complex128)
        nf = (L + 1) * 2 * L
        out = np.zeros(nf, np.float64 if is_real else np.complex128)
        rc = self.lib.orc_inverse(L, lmax, n, int(is_real), _ptr(c.view(np.float64)), _ptr(out.view(np.float64)))
        assert rc == 0
        return out


class Reference:
    """ctypes view of the reference headers compiled in place (_ref)."""

    ALL, NONNEGATIVE, SINGLE = 0, 1, 2

    @staticmethod
    def available() -> bool:
        return os.path.exists(REFERENCE_PATH)

    def __init__(self):
        if not self.available():
            raise FileNotFoundError(REFERENCE_PATH)
        self.lib = ctypes.CDLL(REFERENCE_PATH)
        L = self.lib
        L.ref_grid_create.argtypes = [ctypes.c_int] * 5
        L.ref_grid_create.restype = ctypes.c_void_p
        L.ref_grid_destroy.argtypes = [ctypes.c_void_p]
        L.ref_grid_destroy.restype = None
        L.ref_grid_nodes.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ref_grid_nodes.restype = None
        for f in (L.ref_forward, L.ref_inverse):
            f.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3 + [_dp, _dp]
        L.ref_wigner_block.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp]
        L.ref_wigner_block.restype = ctypes.c_long
        L.ref_wigner_single.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] + [ctypes.c_int] * 2 + [_dp]
        L.ref_wigner_single.restype = ctypes.c_long
        L.ref_roundtrip_batch.argtypes = (
            [ctypes.c_void_p] + [ctypes.c_int] * 4 + [_dp, _dp, _dp] + [ctypes.c_long] * 2 + [ctypes.c_int]
        )
        L.ref_max_threads.restype = ctypes.c_int
        L.ref_chunked_nodes.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.ref_chunked_nodes.restype = None
        _ip = ctypes.POINTER(ctypes.c_int)
        L.ref_chunked_inverse_rings.argtypes = [ctypes.c_int] * 4 + [_dp, ctypes.c_int, _ip, _dp]
        L.ref_chunked_inverse_rings.restype = ctypes.c_int
        L.ref_chunked_forward_orders.argtypes = ([ctypes.c_int] * 4 + [_dp, ctypes.c_int, _ip, ctypes.c_int, _dp])
        L.ref_chunked_forward_orders.restype = ctypes.c_int

    def grid(self, lmax, nmax, mrange=0, nrange=0, long_double=False):
        return RefGrid(self, lmax, nmax, mrange, nrange, long_double)

    def wigner_single(self, lmax, mmax, nmax, theta, four_pi=False, long_double=False):
        n = self.lib.ref_wigner_single(lmax, mmax, nmax, theta, int(four_pi), int(long_double), None)
        out = np.zeros(n)
        self.lib.ref_wigner_single(lmax, mmax, nmax, theta, int(four_pi), int(long_double), _ptr(out))
        return out

    def max_threads(self) -> int:
        return self.lib.ref_max_threads()

    # Transforms at any degree with the reference's Wigner table built on
    # chunks of colatitudes (ref_harness.cpp: ref_chunked_*); long double is
    # the accuracy yardstick, double the reference's own FP64 values.
    def chunked_nodes(self, lmax, long_double=True):
        th = np.zeros(lmax + 1)
        w = np.zeros(lmax + 1)
        self.lib.ref_chunked_nodes(lmax, int(long_double), _ptr(th), _ptr(w))
        return th, w

    def chunked_inverse_rings(self, lmax, n, is_real, coef, rings, long_double=True):
        """InverseTransformation on the listed rings only: array
        [len(rings), 2 lmax] (real or complex)."""
        c = np.ascontiguousarray(coef, dtype=np.complex128)
        r = np.ascontiguousarray(rings, dtype=np.int32)
        out = np.zeros((r.size, 2 * lmax), np.float64 if is_real else np.complex128)
        rc = self.lib.ref_chunked_inverse_rings(
            lmax, n, int(is_real), int(long_double), _ptr(c.view(np.float64)), r.size,
            r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _ptr(out.view(np.float64).reshape(-1)))
        if rc:
            raise ValueError(f"reference chunked inverse rejected (rc={rc})")
        return out

    def chunked_forward_orders(self, lmax, n, is_real, grid, orders, chunk=64, long_double=True):
        """ForwardTransformation restricted to the listed orders:
        {m: c_{l,m} for l = max(|m|,|n|)..lmax}."""
        g = np.ascontiguousarray(grid, dtype=np.float64 if is_real else np.complex128)
        o = np.ascontiguousarray(orders, dtype=np.int32)
        sizes = [lmax - max(abs(int(m)), abs(n)) + 1 for m in o]
        out = np.zeros(sum(sizes), np.complex128)
        rc = self.lib.ref_chunked_forward_orders(
            lmax, n, int(is_real), int(long_double), _ptr(g.view(np.float64).reshape(-1)), o.size,
            o.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), chunk, _ptr(out.view(np.float64)))
        if rc:
            raise ValueError(f"reference chunked forward rejected (rc={rc})")
        res, k = {}, 0
        for m, s in zip(o, sizes):
            res[int(m)] = out[k:k + s]
            k += s
        return res


class RefGrid:
    def __init__(self, ref: Reference, lmax, nmax, mrange, nrange, long_double):
        self.ref = ref
        self.L = lmax
        self.h = ref.lib.ref_grid_create(lmax, nmax, mrange, nrange, int(long_double))
        if not self.h:
            raise ValueError("reference grid creation failed")
        self.n_theta = lmax + 1
        self.n_phi = 2 * lmax

    def close(self):
        if self.h:
            self.ref.lib.ref_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def nodes(self):
        th = np.zeros(self.n_theta)
        w = np.zeros(self.n_theta)
        self.ref.lib.ref_grid_nodes(self.h, _ptr(th), _ptr(w))
        return th, w

    def forward(self, lmax, n, is_real, grid, out=None):
        g = np.ascontiguousarray(grid, dtype=np.float64 if is_real else np.complex128)
        if out is None:
            out = np.zeros(coef_size(lmax, n, is_real), np.complex128)
        rc = self.ref.lib.ref_forward(self.h, lmax, n, int(is_real), _ptr(g.view(np.float64)), _ptr(out.view(np.float64)))
        if rc:
            raise ValueError(f"reference forward rejected (rc={rc})")
        return out

    def inverse(self, lmax, n, is_real, coef):
        c = np.ascontiguousarray(coef, dtype=np.complex128)
        nf = self.n_theta * self.n_phi
        out = np.zeros(nf, np.float64 if is_real else np.complex128)
        rc = self.ref.lib.ref_inverse(self.h, lmax, n, int(is_real), _ptr(c.view(np.float64)), _ptr(out.view(np.float64)))
        if rc:
            raise ValueError(f"reference inverse rejected (rc={rc})")
        return out

    def wigner_block(self, n, itheta):
        k = self.ref.lib.ref_wigner_block(self.h, n, itheta, None)
        if k < 0:
            raise ValueError("bad (n, itheta)")
        out = np.zeros(k)
        self.ref.lib.ref_wigner_block(self.h, n, itheta, _ptr(out))
        return out

    def roundtrip_batch(self, lmax, n, is_real, coefs: np.ndarray, nthreads: int):
        """Inverse then forward per field (OpenMP over fields); returns coefs."""
        nf = coefs.shape[0]
        cs = coef_size(lmax, n, is_real)
        fs = self.n_theta * self.n_phi
        cin = np.ascontiguousarray(coefs, dtype=np.complex128)
        cout = np.zeros_like(cin)
        scratch = np.zeros(nf * fs * (1 if is_real else 2))
        rc = self.ref.lib.ref_roundtrip_batch(
            self.h, lmax, n, int(is_real), nf,
            _ptr(cin.view(np.float64).reshape(-1)), _ptr(cout.view(np.float64).reshape(-1)),
            _ptr(scratch), cs, fs, nthreads,
        )
        if rc:
            raise ValueError("reference batch failed")
        return cout


def random_coefficients(rng: np.random.Generator, L_grid: int, lmax: int, n: int,
                        is_real: bool, envelope: Optional[float] = None) -> np.ndarray:
    """Seeded coefficients with the reference fixture semantics.

    Complex fields: N(0,1) + i N(0,1), and c_{L,L} = 0 when lmax equals the
    grid degree (GridBase.h:124-140). Real fields: the same, with
    Im c_{l,0} = 0 for every l and Im c_{L,L} = 0 when lmax equals the grid
    degree (GridBase.h:151-172). ``envelope`` p multiplies degree l by
    (l+1)^-p (the power-law envelopes of the benchmark workloads).
    """
    size = coef_size(lmax, n, is_real)
    c = rng.standard_normal(size) + 1j * rng.standard_normal(size)
    ls, ms = degree_order(lmax, n, is_real)
    if envelope is not None:
        c = c * (ls + 1.0) ** (-envelope)
    if is_real:
        c[ms == 0] = c[ms == 0].real
        if lmax == L_grid:
            c[-1] = c[-1].real
    elif lmax == L_grid:
        c[-1] = 0
    return c


def degree_order(lmax: int, n: int, is_real: bool):
    """(l, m) for every slot of the GSHIndices<All|NonNegative> layout."""
    ls, ms = [], []
    for l in range(abs(n), lmax + 1):
        mr = range(0, l + 1) if is_real else range(-l, l + 1)
        ls.extend([l] * len(mr))
        ms.extend(mr)
    return np.asarray(ls), np.asarray(ms)
