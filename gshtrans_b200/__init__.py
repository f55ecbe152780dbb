"""gshtrans_b200 — Gauss-Legendre generalized-spherical-harmonic transforms on B200.

Python mirror of the reference's ``GaussLegendreGrid`` interface
(GaussLegendreGrid.h:24-321, GridBase.h:13-177) over the C ABI of
``libgsht_cuda.so`` (include/gsht.h). Method names, argument meaning and the
forward transform's accumulate-into-output semantics follow the reference;
where the reference asserts, this layer raises :class:`BadArgument`.

Buffers may be NumPy arrays (host) or PyTorch tensors (host or CUDA); CUDA
tensors are used in place and the call only enqueues work on the current
stream. The CUDA library is required: there is no CPU fallback, and importing
this package raises if ``libgsht_cuda.so`` cannot be loaded.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

__all__ = [
    "All", "NonNegative", "Single", "FP64", "BF16X3", "OZAKI", "RECURRENCE", "OZAKI4",
    "STAGES", "StageProfile",
    "GaussLegendreGrid", "GSHTError", "BadArgument", "library", "launch_count",
    "coefficient_size", "wigner", "Batch", "random_coefficients", "degree_order",
    "set_allocator", "use_torch_allocator", "alloc_stats",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgsht_cuda.so")

# Index ranges (Concepts.h:24-27) and precision forms (include/gsht.h).
All, NonNegative, Single = 0, 1, 2
FP64, BF16X3, OZAKI, RECURRENCE, OZAKI4 = 0, 1, 2, 3, 4
_FORM_BIT = {FP64: 1, BF16X3: 2, OZAKI: 4, RECURRENCE: 8, OZAKI4: 4}
_PRECISION_NAMES = {"fp64": FP64, "bf16x3": BF16X3, "ozaki": OZAKI, "recurrence": RECURRENCE,
                    "ozaki4": OZAKI4}

_STATUS = {
    0: "OK", 1: "BAD_ARG", 2: "OOM", 3: "CUDA_ERROR", 4: "TIMEOUT",
    5: "UNSUPPORTED", 6: "NO_DEVICE",
}


class GSHTError(RuntimeError):
    """A non-OK status from libgsht_cuda.so."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


class BadArgument(GSHTError, ValueError):
    """Invalid arguments (the reference asserts on these)."""


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python gshtrans_b200/build.py`"
        )
    lib = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    lib.gsht_grid_create.argtypes = [ip, ip, ip, ip, ctypes.c_uint, ctypes.POINTER(vp)]
    lib.gsht_grid_destroy.argtypes = [vp]
    lib.gsht_grid_shape.argtypes = [vp] + [ctypes.POINTER(ip)] * 5
    lib.gsht_grid_nodes.argtypes = [vp, dp, dp]
    lib.gsht_wigner_block.argtypes = [vp, ip, ip, dp, ctypes.POINTER(ctypes.c_long)]
    lib.gsht_wigner_compute.argtypes = [ip] * 7 + [dp, ip, dp, ctypes.POINTER(ctypes.c_long)]
    lib.gsht_coefficient_size.argtypes = [ip, ip, ip]
    lib.gsht_coefficient_size.restype = ctypes.c_long
    for f in (lib.gsht_forward, lib.gsht_inverse):
        f.argtypes = [vp, ip, ip, ip, ip, vp, vp, vp]
    for f in (lib.gsht_forward_batch, lib.gsht_inverse_batch):
        f.argtypes = [vp, ip, ip, ip, ip, ip, vp, vp, vp]
    lib.gsht_device_status.argtypes = [vp]
    lib.gsht_profile_enable.argtypes = [ip]
    lib.gsht_profile_read.argtypes = [vp, vp, ip]
    lib.gsht_last_error.restype = ctypes.c_char_p
    lib.gsht_launch_count.restype = ctypes.c_ulonglong
    lib.gsht_check_bounded_wait.argtypes = [vp, vp]
    lib.gsht_set_allocator.argtypes = [_ALLOC_FN, _FREE_FN, vp]
    lib.gsht_alloc_stats.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)] * 2 + [ctypes.POINTER(ctypes.c_size_t)]
    return lib


# gsht_alloc_fn / gsht_free_fn (include/gsht.h)
_ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
_FREE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p)


library = _load()


def launch_count() -> int:
    """Kernels launched by libgsht_cuda.so in this process."""
    return int(library.gsht_launch_count())


_allocator_refs = None  # keeps the ctypes callbacks of the current hook alive


def set_allocator(alloc=None, free=None):
    """Routes every device allocation of the library through ``alloc(bytes)
    -> int pointer (0 on failure)`` and ``free(pointer)`` (gsht_set_allocator;
    no counterpart in the reference). ``set_allocator()`` restores
    cudaMalloc / cudaFree. A pointer is released by the hook that made it, so
    the callables of an earlier hook stay referenced here while it may still
    own memory."""
    global _allocator_refs
    if (alloc is None) != (free is None):
        raise BadArgument(1, "give both alloc and free, or neither")
    if alloc is None:
        _check(library.gsht_set_allocator(_ALLOC_FN(), _FREE_FN(), None))
        return

    def _alloc(nbytes, _ctx):
        try:
            return int(alloc(int(nbytes)) or 0)
        except Exception:
            return 0

    def _free(ptr, _ctx):
        try:
            free(int(ptr))
        except Exception:
            pass

    refs = (_ALLOC_FN(_alloc), _FREE_FN(_free))
    _check(library.gsht_set_allocator(refs[0], refs[1], None))
    _old_allocators.append(_allocator_refs)
    _allocator_refs = refs


_old_allocators = []


def use_torch_allocator():
    """Draws the library's device memory from PyTorch's caching allocator on
    the current device (torch.cuda.caching_allocator_alloc / _delete)."""
    import torch

    set_allocator(lambda n: torch.cuda.caching_allocator_alloc(n),
                  lambda p: torch.cuda.caching_allocator_delete(p))


def alloc_stats():
    """(allocations, releases, live bytes) of the library's device memory in
    this process (gsht_alloc_stats)."""
    a, r = ctypes.c_ulonglong(), ctypes.c_ulonglong()
    b = ctypes.c_size_t()
    _check(library.gsht_alloc_stats(ctypes.byref(a), ctypes.byref(r), ctypes.byref(b)))
    return int(a.value), int(r.value), int(b.value)


STAGES = ("prep_inverse", "legendre_inverse", "fft_inverse", "fft_forward",
          "prep_forward", "legendre_forward", "accumulate_forward")


class StageProfile:
    """Per-stage device time of the transform calls made inside a ``with``
    block (gsht_profile_enable / gsht_profile_read: CUDA events around every
    stage of direct calls; captured graphs are not timed). After the block,
    ``stages`` maps each stage name to ``(milliseconds, kernel launches)``.
    No counterpart in the reference, which has no tracing."""

    def __enter__(self):
        _check(library.gsht_profile_enable(1))
        self.stages = {}
        return self

    def __exit__(self, *exc):
        n = len(STAGES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_long * n)()
        try:
            _check(library.gsht_profile_read(ctypes.cast(ms, ctypes.c_void_p),
                                             ctypes.cast(cnt, ctypes.c_void_p), n))
        finally:
            library.gsht_profile_enable(0)
        self.stages = {name: (ms[i], int(cnt[i])) for i, name in enumerate(STAGES)}
        return False


library.gsht_tc_trace_enable.argtypes = [ctypes.c_int]
library.gsht_tc_trace_read.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
TRACE_SLOTS = ("producer", "producer_wait_free_stage", "mma", "mma_wait_loaded_stage",
               "mma_wait_epilogue", "epilogue", "epilogue_wait_accumulators", "ctas", "mma_ctas")


class TensorCoreTrace:
    """Per-role cycle trace of the tensor-core Legendre kernels launched
    inside a ``with`` block (gsht_tc_trace_enable / gsht_tc_trace_read: the
    traced kernel copies time every pipeline wait with clock64). ``read(form,
    direction)`` returns the last traced launch's counters as a dict of
    TRACE_SLOTS, plus per-role fractions: the share of the MMA issuer's time
    spent waiting for loaded stages and for the epilogue, and the rest, during
    which it issues MMAs. No counterpart in the reference."""

    def __enter__(self):
        _check(library.gsht_tc_trace_enable(1))
        return self

    def __exit__(self, *exc):
        library.gsht_tc_trace_enable(0)
        return False

    @staticmethod
    def read(form="bf16x3", direction=0):
        out = (ctypes.c_double * len(TRACE_SLOTS))()
        _check(library.gsht_tc_trace_read(_precision(form), int(direction),
                                          ctypes.cast(out, ctypes.c_void_p), len(TRACE_SLOTS)))
        c = {name: out[i] for i, name in enumerate(TRACE_SLOTS)}
        if c["mma"] > 0:
            c["mma_frac_wait_loaded_stage"] = c["mma_wait_loaded_stage"] / c["mma"]
            c["mma_frac_wait_epilogue"] = c["mma_wait_epilogue"] / c["mma"]
            c["mma_frac_issuing"] = 1.0 - c["mma_frac_wait_loaded_stage"] - c["mma_frac_wait_epilogue"]
        if c["producer"] > 0:
            c["producer_frac_wait_free_stage"] = c["producer_wait_free_stage"] / c["producer"]
        if c["epilogue"] > 0:
            c["epilogue_frac_wait_accumulators"] = c["epilogue_wait_accumulators"] / c["epilogue"]
        return c


def _check(status: int):
    if status != 0:
        msg = library.gsht_last_error().decode()
        if status == 1:
            raise BadArgument(status, msg)
        raise GSHTError(status, msg)


def wigner(lmax: int, mmax: int, nmax: int, theta, mrange: int = All, nrange: int = Single,
           four_pi: bool = False, row_major: bool = False) -> np.ndarray:
    """Wigner<double, Norm, MRange, NRange, AngleRange, Storage>(lMax, mMax,
    nMax, theta) (Wigner.h:99-159): the values for every (n, angle) block in
    the reference's storage order, computed on the GPU."""
    th = np.ascontiguousarray(np.atleast_1d(np.asarray(theta, dtype=np.float64)))
    dp = ctypes.POINTER(ctypes.c_double)
    cnt = ctypes.c_long()
    args = (lmax, mmax, nmax, mrange, nrange, int(four_pi), int(row_major), th.ctypes.data_as(dp), th.size)
    _check(library.gsht_wigner_compute(*args, None, ctypes.byref(cnt)))
    out = np.zeros(cnt.value)
    _check(library.gsht_wigner_compute(*args, out.ctypes.data_as(dp), ctypes.byref(cnt)))
    return out


def degree_order(lmax: int, n: int, is_real: bool):
    """Degree and order of every slot of the packed layout, GSHIndices<All>
    (complex) or GSHIndices<NonNegative> (real) (Indexing.h:104-131)."""
    ls = np.arange(abs(n), lmax + 1)
    width = ls + 1 if is_real else 2 * ls + 1
    l_of = np.repeat(ls, width)
    start = np.repeat(np.cumsum(width) - width, width)
    pos = np.arange(l_of.size) - start
    m_of = pos if is_real else pos - l_of
    return l_of, m_of


def random_coefficients(rng, grid_lmax: int, lmax: int, n: int, is_real: bool,
                        envelope=None) -> np.ndarray:
    """GridBase::RandomComplexCoefficient / RandomRealCoefficient
    (GridBase.h:124-172) from a NumPy generator: N(0,1) + i N(0,1) per slot
    (real parts drawn first), times (l+1)^-envelope if given; complex fields
    get c_{L,L} = 0 and real fields Im c_{l,0} = 0 and Im c_{L,L} = 0 when
    lmax equals the grid degree L."""
    size = coefficient_size(lmax, n, is_real)
    c = rng.standard_normal(size) + 1j * rng.standard_normal(size)
    ls, ms = degree_order(lmax, n, is_real)
    if envelope is not None:
        c = c * (ls + 1.0) ** (-float(envelope))
    if is_real:
        c[ms == 0] = c[ms == 0].real
        if lmax == grid_lmax:
            c[-1] = c[-1].real
    elif lmax == grid_lmax:
        c[-1] = 0
    return c


def coefficient_size(lmax: int, n: int, is_real: bool) -> int:
    """GridBase::RealCoefficientSize / ComplexCoefficientSize (GridBase.h:79-85)."""
    s = library.gsht_coefficient_size(lmax, n, int(is_real))
    if s < 0:
        raise BadArgument(1, f"no coefficients for lmax={lmax}, n={n}")
    return int(s)


def _precision(p) -> int:
    if isinstance(p, str):
        return _PRECISION_NAMES[p.lower()]
    return int(p)


def _buffer(x):
    """(pointer, is_complex, numel, writable-object) for a NumPy array or torch tensor."""
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise BadArgument(1, "arrays must be C-contiguous")
        if x.dtype == np.complex128:
            return x.ctypes.data, True, x.size
        if x.dtype == np.float64:
            return x.ctypes.data, False, x.size
        raise BadArgument(1, f"unsupported dtype {x.dtype}")
    try:
        import torch
    except ImportError:  # pragma: no cover
        torch = None
    if torch is not None and isinstance(x, torch.Tensor):
        if not x.is_contiguous():
            raise BadArgument(1, "tensors must be contiguous")
        if x.dtype == torch.complex128:
            return x.data_ptr(), True, x.numel()
        if x.dtype == torch.float64:
            return x.data_ptr(), False, x.numel()
        raise BadArgument(1, f"unsupported dtype {x.dtype}")
    raise BadArgument(1, f"unsupported buffer type {type(x)}")


def _current_stream(*bufs) -> Optional[int]:
    for b in bufs:
        if not isinstance(b, np.ndarray):
            import torch

            if b.is_cuda:
                return torch.cuda.current_stream(b.device).cuda_stream
    return None


class GaussLegendreGrid:
    """GaussLegendreGrid<double, MRange, NRange>(lMax, nMax) on the GPU.

    ``mrange`` is ``All`` or ``NonNegative``; ``nrange`` is ``All``,
    ``NonNegative`` or ``Single`` (GaussLegendreGrid.h:24-26). ``forms``
    selects which table forms are built besides FP64: any of ``"bf16x3"``,
    ``"ozaki"``, ``"recurrence"``. ``forms=("recurrence",)`` alone stores no
    table: every transform runs in FP64 with the Wigner values generated by
    the l-recurrence inside the contraction (precision ``"fp64"`` or
    ``"recurrence"``).
    """

    def __init__(self, lmax: int, nmax: int, mrange: int = All, nrange: int = All,
                 forms=()):
        mask = 0
        for f in forms:
            mask |= _FORM_BIT[_precision(f)]
        if mask != _FORM_BIT[RECURRENCE]:
            mask |= _FORM_BIT[FP64]
        h = ctypes.c_void_p()
        _check(library.gsht_grid_create(int(lmax), int(nmax), int(mrange), int(nrange),
                                        mask, ctypes.byref(h)))
        self._h = h
        self._mrange = mrange
        self._nrange = nrange
        vals = [ctypes.c_int() for _ in range(5)]
        _check(library.gsht_grid_shape(h, *[ctypes.byref(v) for v in vals]))
        self._lmax, self._nmax, self._min_n, self._nt, self._np = (v.value for v in vals)

    def close(self):
        if getattr(self, "_h", None):
            library.gsht_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- geometry (GaussLegendreGrid.h:86-103, GridBase.h:17-114) ----
    def MaxDegree(self) -> int:
        return self._lmax

    def MaxUpperIndex(self) -> int:
        return self._nmax

    def MinUpperIndex(self) -> int:
        return self._min_n

    def UpperIndices(self):
        return range(self._min_n, self._nmax + 1)

    def NumberOfCoLatitudes(self) -> int:
        return self._nt

    def NumberOfLongitudes(self) -> int:
        return self._np

    def FieldSize(self) -> int:
        return self._nt * self._np

    def CoLatitudes(self) -> np.ndarray:
        th = np.zeros(self._nt)
        _check(library.gsht_grid_nodes(self._h, th.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None))
        return th

    def CoLatitudeWeights(self) -> np.ndarray:
        w = np.zeros(self._nt)
        _check(library.gsht_grid_nodes(self._h, None, w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return w

    def Longitudes(self) -> np.ndarray:
        return np.arange(self._np) * (2 * np.pi / self._np)

    def LongitudeWeights(self) -> np.ndarray:
        return np.full(self._np, 2 * np.pi / self._np)

    def RealCoefficientSize(self, lmax: int, n: int) -> int:
        return coefficient_size(lmax, n, True)

    def ComplexCoefficientSize(self, lmax: int, n: int) -> int:
        return coefficient_size(lmax, n, False)

    def CoefficientSize(self, lmax: int, n: int) -> int:
        return coefficient_size(lmax, n, False)

    def CoefficientSizeNonNegative(self, lmax: int, n: int) -> int:
        return coefficient_size(lmax, n, True)

    def Wigner(self, n: int, itheta: int) -> np.ndarray:
        """Table block d^l_{mn}(theta_itheta) in the reference layout (Wigner.h:241-244)."""
        cnt = ctypes.c_long()
        _check(library.gsht_wigner_block(self._h, n, itheta, None, ctypes.byref(cnt)))
        out = np.zeros(cnt.value)
        _check(library.gsht_wigner_block(self._h, n, itheta,
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         ctypes.byref(cnt)))
        return out

    def device_status(self):
        """Synchronises and raises GSHTError(TIMEOUT) if a kernel gave up a bounded wait."""
        _check(library.gsht_device_status(self._h))

    def check_bounded_wait(self, stream=None):
        """Enqueues gsht_check_bounded_wait: a wait that nothing completes runs
        to its limit (about half a second) and raises this grid's device error
        word; the next device_status() raises GSHTError(TIMEOUT)."""
        _check(library.gsht_check_bounded_wait(self._h, stream))

    # ---- transforms (GaussLegendreGrid.h:108-321) ----
    def ForwardTransformation(self, lmax: int, n: int, in_, out, precision="fp64"):
        """Grid values -> coefficients, ACCUMULATED into ``out``."""
        self._transform(0, lmax, n, in_, out, precision, 1)
        return out

    def InverseTransformation(self, lmax: int, n: int, in_, out, precision="fp64"):
        """Coefficients -> grid values (``out`` overwritten)."""
        self._transform(1, lmax, n, in_, out, precision, 1)
        return out

    def forward_batch(self, lmax: int, n: int, in_, out, precision="fp64"):
        """Batched forward: ``in_`` holds count fields back to back."""
        return self._transform(0, lmax, n, in_, out, precision, None)

    def inverse_batch(self, lmax: int, n: int, in_, out, precision="fp64"):
        """Batched inverse: ``in_`` holds count coefficient vectors back to back."""
        return self._transform(1, lmax, n, in_, out, precision, None)

    def _transform(self, direction, lmax, n, in_, out, precision, count):
        pin, cin, nin = _buffer(in_)
        pout, cout, nout = _buffer(out)
        grid_complex = cin if direction == 0 else cout
        coef_ok = (cout if direction == 0 else cin)
        if not coef_ok:
            raise BadArgument(1, "coefficients must be complex128")
        is_real = not grid_complex
        if self._mrange != All and not is_real:
            raise BadArgument(1, "complex fields need MRange = All")
        if abs(n) > lmax or lmax < 0 or lmax > self._lmax:
            raise BadArgument(1, f"bad (lmax={lmax}, n={n}) for grid degree {self._lmax}")
        cs = coefficient_size(lmax, n, is_real)
        fs = self.FieldSize()
        n_grid = nin if direction == 0 else nout
        n_coef = nout if direction == 0 else nin
        if count is None:
            if fs == 0 or n_grid % fs or n_coef % cs or n_grid // fs != n_coef // cs:
                raise BadArgument(1, "batch buffers do not hold a whole number of fields")
            count = n_grid // fs
        elif n_grid != fs or n_coef != cs:
            raise BadArgument(1, f"sizes: grid {n_grid} (want {fs}), coefficients {n_coef} (want {cs})")
        stream = _current_stream(in_, out)
        fn = library.gsht_forward_batch if direction == 0 else library.gsht_inverse_batch
        _check(fn(self._h, lmax, n, int(is_real), _precision(precision), count,
                  ctypes.c_void_p(pin), ctypes.c_void_p(pout),
                  ctypes.c_void_p(stream) if stream else None))
        return out


class _FieldDesc(ctypes.Structure):
    _fields_ = [("lmax", ctypes.c_int), ("n", ctypes.c_int), ("is_real", ctypes.c_int),
                ("coef_in", ctypes.c_void_p), ("grid", ctypes.c_void_p),
                ("coef_out", ctypes.c_void_p)]


library.gsht_plan_batch.argtypes = [ctypes.POINTER(_FieldDesc), ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
library.gsht_batch_execute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
library.gsht_batch_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_long)]
library.gsht_batch_group.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 5
library.gsht_batch_schedule.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
library.gsht_batch_destroy.argtypes = [ctypes.c_void_p]

BATCH_FORWARD, BATCH_INVERSE, BATCH_ROUND_TRIP = 0, 1, 2


class Batch:
    """Many fields of uneven lmax / upper index / kind, transformed by one CUDA
    graph launch per call (``gsht_plan_batch``; no reference counterpart: the
    reference transforms one field per call, GaussLegendreGrid.h:108-321).

    ``fields`` is a list of ``(lmax, n, is_real, coef_in, grid, coef_out)``
    with CUDA tensors in the layouts of the single-field transforms (each
    field on its own grid, nTheta = lmax + 1, nPhi = 2 lmax). ``inverse()``
    writes the grids from ``coef_in``; ``forward()`` adds the grids'
    coefficients into ``coef_out``; ``round_trip()`` does both. The tensors
    must stay alive (and in place) for the life of the plan.
    """

    def __init__(self, fields, precision="bf16x3", autotune=True):
        descs = []
        self._keep = []
        for lmax, n, is_real, cin, grid, cout in fields:
            for t in (cin, grid, cout):
                if not getattr(t, "is_cuda", False):
                    raise BadArgument(1, "batch buffers must be CUDA tensors")
                self._keep.append(t)
            descs.append(_FieldDesc(int(lmax), int(n), int(bool(is_real)), cin.data_ptr(),
                                    grid.data_ptr(), cout.data_ptr()))
        arr = (_FieldDesc * len(descs))(*descs)
        h = ctypes.c_void_p()
        _check(library.gsht_plan_batch(arr, len(descs), _precision(precision), int(bool(autotune)),
                                       ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            library.gsht_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover
            pass

    def _run(self, mode):
        import torch

        _check(library.gsht_batch_execute(self._h, mode,
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    def forward(self):
        self._run(BATCH_FORWARD)

    def inverse(self):
        self._run(BATCH_INVERSE)

    def round_trip(self):
        self._run(BATCH_ROUND_TRIP)

    def streams(self) -> int:
        """Streams the plan's graphs spread the groups over (gsht_batch_schedule)."""
        k = ctypes.c_int()
        _check(library.gsht_batch_schedule(self._h, ctypes.byref(k)))
        return k.value

    def info(self):
        """(groups, grids, graph nodes per mode [forward, inverse, round trip])."""
        g, d = ctypes.c_int(), ctypes.c_int()
        nodes = (ctypes.c_long * 3)()
        _check(library.gsht_batch_info(self._h, ctypes.byref(g), ctypes.byref(d), nodes))
        return g.value, d.value, list(nodes)

    def groups(self):
        """[(lmax, n, is_real, count, tile width)] per group."""
        g, _, _ = self.info()
        out = []
        for i in range(g):
            v = [ctypes.c_int() for _ in range(5)]
            _check(library.gsht_batch_group(self._h, i, *[ctypes.byref(x) for x in v]))
            out.append(tuple(x.value for x in v))
        return out
