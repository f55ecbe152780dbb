"""Canonical-component fields and their fused pointwise expressions.

Python mirror of the reference's ``CanonicalComponentField<N, Grid, Value>``
(CanonicalComponentField.h:39-125) and its lazy expression nodes
(CanonicalComponentFieldBinary.h:100-305, CanonicalComponentFieldUnary.h
:103-354, CanonicalComponentFieldOverloads.h:22-262). Building an expression
allocates nothing; assigning it (``out.assign(expr)``, or ``expr.evaluate()``)
flattens the node tree into a postfix program and evaluates every grid point
in one kernel (``gsht_field_eval``), reading each input once.

Upper-index bookkeeping follows the reference's types: ``u * v`` carries
N0 + N1; ``+`` and ``-`` need equal N; ``/`` needs the divisor's N == 0;
``conj`` keeps N (CanonicalComponentFieldUnary.h:104-107, which is what the
reference does even though conjugation maps n to -n mathematically), so an
explicit ``upper_index=`` may be given when assigning.

Fields hold their values in a torch tensor on the GPU, ring-major
(nTheta x nPhi) as the reference stores them; ``Data()`` returns that
tensor, ready for ``GaussLegendreGrid`` transforms.
"""

from __future__ import annotations

import ctypes
from typing import List, Tuple

from . import BadArgument, _check, library

_OP = dict(LOAD=0, CONST=1, ADD=2, SUB=3, MUL=4, DIV=5, NEG=6, CONJ=7, REAL=8, IMAG=9)


class _Op(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("arg", ctypes.c_int),
                ("re", ctypes.c_double), ("im", ctypes.c_double)]


library.gsht_field_eval.argtypes = [
    ctypes.POINTER(_Op), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
    ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
    ctypes.c_long, ctypes.c_int, ctypes.c_long, ctypes.c_void_p,
]
library.gsht_field_jit_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p]


def jit_stats():
    """(programs compiled into kernels of their own, programs that could not
    be and run interpreted) so far in this process (gsht_field_jit_stats)."""
    c, f = ctypes.c_int(), ctypes.c_int()
    _check(library.gsht_field_jit_stats(ctypes.byref(c), ctypes.byref(f)))
    return int(c.value), int(f.value)


class Expr:
    """A lazy pointwise expression over fields of one grid."""

    N: int
    is_real: bool

    # --- building -----------------------------------------------------------
    def __add__(self, o):
        return _binary("ADD", self, o)

    def __radd__(self, o):
        return _binary("ADD", _const(o, self), self)

    def __sub__(self, o):
        return _binary("SUB", self, o)

    def __rsub__(self, o):
        return _binary("SUB", _const(o, self), self)

    def __mul__(self, o):
        return _binary("MUL", self, o)

    def __rmul__(self, o):
        return _binary("MUL", _const(o, self), self)

    def __truediv__(self, o):
        return _binary("DIV", self, o)

    def __neg__(self):
        return _Unary("NEG", self, self.N, self.is_real)

    # --- flattening ---------------------------------------------------------
    def _emit(self, ops: List[Tuple[int, int, complex]], inputs: list):
        raise NotImplementedError

    def fields(self):
        raise NotImplementedError

    def evaluate(self, upper_index=None):
        """Materialise into a new field (CanonicalComponentField(grid) then =)."""
        g, count = self._geometry()
        out = Field(g, self.N if upper_index is None else upper_index, self.is_real, count=count)
        out.assign(self, upper_index=upper_index)
        return out

    def _geometry(self):
        fs = self.fields()
        if not fs:
            raise BadArgument(1, "an expression needs at least one field")
        g, count = fs[0].grid, fs[0].count
        for f in fs:
            if f.grid is not g or f.count != count:
                raise BadArgument(1, "expression mixes grids or batch sizes")
        return g, count


def conj(u: Expr, upper_index=None) -> Expr:
    """CanonicalComponentFieldConj. Like the reference it keeps the upper
    index by default (CanonicalComponentFieldUnary.h:104-107); pass
    ``upper_index=-u.N`` for the mathematically conjugate index, which makes
    expressions such as ``u*v + conj(u, -1)*u`` (u: n=+1, v: n=-1) well typed."""
    n = u.N if upper_index is None else int(upper_index)
    return _Unary("CONJ", u, n, u.is_real) if not u.is_real else u


def real(u: Expr) -> Expr:
    """CanonicalComponentFieldReal (real-valued result)."""
    return _Unary("REAL", u, u.N, True)


def imag(u: Expr) -> Expr:
    """CanonicalComponentFieldImag (real-valued result; zero for real fields)."""
    return _Unary("IMAG", u, u.N, True)


def _const(c, like: Expr) -> "_Const":
    return _Const(complex(c), like.is_real and not isinstance(c, complex))


def _binary(op, a, b):
    if not isinstance(b, Expr):
        # Scalar forms (CanonicalComponentFieldOverloads.h:66-146): + and - only
        # for N == 0 fields, * and / for any N.
        if op in ("ADD", "SUB") and a.N != 0:
            raise BadArgument(1, "scalar + and - need upper index 0")
        b = _const(b, a)
        return _Binary(op, a, b, a.N, a.is_real and b.is_real)
    if a.is_real != b.is_real:
        raise BadArgument(1, "operands must have the same value type")
    if op in ("ADD", "SUB"):
        if a.N != b.N:
            raise BadArgument(1, f"{op.lower()} needs equal upper indices ({a.N} vs {b.N})")
        n = a.N
    elif op == "MUL":
        n = a.N + b.N
    else:
        if b.N != 0:
            raise BadArgument(1, "division needs a divisor of upper index 0")
        n = a.N
    return _Binary(op, a, b, n, a.is_real)


class _Const(Expr):
    def __init__(self, c: complex, is_real: bool):
        self.c, self.N, self.is_real = c, 0, is_real

    def _emit(self, ops, inputs):
        ops.append((_OP["CONST"], 0, self.c))

    def fields(self):
        return []


class _Unary(Expr):
    def __init__(self, op, u, n, is_real):
        self.op, self.u, self.N, self.is_real = op, u, n, is_real

    def _emit(self, ops, inputs):
        self.u._emit(ops, inputs)
        ops.append((_OP[self.op], 0, 0j))

    def fields(self):
        return self.u.fields()


class _Binary(Expr):
    def __init__(self, op, a, b, n, is_real):
        self.op, self.a, self.b, self.N, self.is_real = op, a, b, n, is_real

    def _emit(self, ops, inputs):
        self.a._emit(ops, inputs)
        self.b._emit(ops, inputs)
        ops.append((_OP[self.op], 0, 0j))

    def fields(self):
        return self.a.fields() + self.b.fields()


class Field(Expr):
    """CanonicalComponentField<N, Grid, RealValued|ComplexValued> on the GPU.

    ``count`` > 1 holds a batch of fields of the same kind back to back (the
    layout the batched transforms use); expressions then act field-wise.
    """

    def __init__(self, grid, n: int, is_real: bool = False, count: int = 1, data=None):
        import torch

        self.grid, self.N, self.is_real, self.count = grid, int(n), bool(is_real), int(count)
        dt = torch.float64 if is_real else torch.complex128
        shape = (count, grid.FieldSize()) if count > 1 else (grid.FieldSize(),)
        if data is None:
            self._data = torch.zeros(shape, dtype=dt, device="cuda")
        else:
            if data.dtype != dt or data.numel() != count * grid.FieldSize() or not data.is_cuda:
                raise BadArgument(1, "data must be a CUDA tensor of the field's kind and size")
            self._data = data.contiguous().view(shape)

    def Data(self):
        """Ring-major values (CanonicalComponentField.h:74)."""
        return self._data

    def UpperIndex(self) -> int:
        return self.N

    def _emit(self, ops, inputs):
        for i, f in enumerate(inputs):
            if f is self:
                ops.append((_OP["LOAD"], i, 0j))
                return
        inputs.append(self)
        ops.append((_OP["LOAD"], len(inputs) - 1, 0j))

    def fields(self):
        return [self]

    def assign(self, expr: Expr, upper_index=None):
        """``*this = expr`` (CanonicalComponentFieldBase.h:201-211), fused."""
        import torch

        if isinstance(expr, (int, float, complex)):
            expr = _Const(complex(expr), self.is_real)
        n = expr.N if upper_index is None else upper_index
        if upper_index is None and not isinstance(expr, _Const) and n != self.N:
            raise BadArgument(1, f"upper index {n} assigned to a field of upper index {self.N}")
        for f in expr.fields():
            if f.grid is not self.grid or f.count != self.count:
                raise BadArgument(1, "expression and target differ in grid or batch size")
        ops, inputs = [], []
        expr._emit(ops, inputs)
        prog = (_Op * len(ops))(*[_Op(o, a, c.real, c.imag) for o, a, c in ops])
        ptrs = (ctypes.c_void_p * max(1, len(inputs)))(*[f._data.data_ptr() for f in inputs])
        kinds = (ctypes.c_int * max(1, len(inputs)))(*[int(f.is_real) for f in inputs])
        fs = self.grid.FieldSize()
        stream = torch.cuda.current_stream().cuda_stream
        _check(library.gsht_field_eval(prog, len(ops), ptrs, kinds, len(inputs),
                                       ctypes.c_void_p(self._data.data_ptr()), int(self.is_real),
                                       fs, self.count, fs, ctypes.c_void_p(stream)))
        return self

    # compound assignments (CanonicalComponentFieldBase.h:222-339)
    def __iadd__(self, o):
        return self.assign(self + o, upper_index=self.N)

    def __isub__(self, o):
        return self.assign(self - o, upper_index=self.N)

    def __imul__(self, o):
        return self.assign(self * o, upper_index=self.N)

    def __itruediv__(self, o):
        return self.assign(self / o, upper_index=self.N)
