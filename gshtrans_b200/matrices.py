"""Matrix fields in canonical components, and their expansions.

Python mirror of the reference's (header-disabled) matrix-field layer
(src/MatrixFieldOld/MatrixField.h, MatrixFieldExpressions.h,
MatrixFieldOverloads.h, IsotropicMatrixField.h): nine canonical components
A_{alpha beta}, alpha, beta in -1, 0, +1, each a CanonicalComponentField of
upper index alpha + beta, stored in one CUDA tensor [9][count][nTheta * nPhi]
with component (alpha, beta) at 3 (alpha + 1) + (beta + 1) (the reference's
Offset, MatrixField.h:97-99). Every pointwise operation is one fused
gsht_field_eval pass per output component; every transform is one batched
call per component (upper indices -2..2, so the grid needs nMax >= 2).

Contractions use the canonical metric (g^{-1,+1} = g^{+1,-1} = -1,
g^{00} = 1), as the reference's complex branch writes them:
  (A u)_alpha = -A_{alpha,-1} u_{+1} + A_{alpha,0} u_0 - A_{alpha,+1} u_{-1}
      (MatrixFieldAction, MatrixFieldExpressions.h:431-436)
  (A B)_{alpha beta} = -A_{alpha,+1} B_{-1,beta} + A_{alpha,0} B_{0,beta}
                       - A_{alpha,-1} B_{+1,beta}   (:509-513)
  det A as the cofactor expansion of MatrixFieldDeterminant (:359-369).
Two reference expressions are corrected here and say so: the negation
returns -A_{alpha beta} (the reference returns -A_{-alpha,-beta},
MatrixFieldExpressions.h:42), and the trace is
-A_{-1,+1} + A_{00} - A_{+1,-1} (the reference's second term reads
A_{+1,+1}, :325). Complex-valued components only (the real-valued branch of
the reference works on a different, real basis).
"""

from __future__ import annotations

from . import BadArgument
from . import fields as F
from .expansions import Expansion
from .fields import Field
from .vectors import CANONICAL_INDICES, VectorField

PAIRS = [(a, b) for a in CANONICAL_INDICES for b in CANONICAL_INDICES]


def _slot(alpha: int, beta: int) -> int:
    if alpha not in CANONICAL_INDICES or beta not in CANONICAL_INDICES:
        raise BadArgument(1, f"canonical indices ({alpha}, {beta}) not in -1, 0, +1")
    return 3 * (alpha + 1) + (beta + 1)


class MatrixField:
    """MatrixField<Grid, ComplexValued> on the GPU: components A_{alpha beta}."""

    def __init__(self, grid, count: int = 1, data=None):
        import torch

        self.grid, self.count = grid, int(count)
        fs = grid.FieldSize()
        if grid.MaxUpperIndex() < 2 or grid.MinUpperIndex() > -2:
            raise BadArgument(1, "matrix fields need a grid with upper indices -2..2")
        if data is None:
            self._data = torch.zeros((9, count, fs), dtype=torch.complex128, device="cuda")
        else:
            if data.dtype != torch.complex128 or data.numel() != 9 * count * fs or not data.is_cuda:
                raise BadArgument(1, "data must be a complex128 CUDA tensor of 9 x count fields")
            self._data = data.contiguous().view(9, count, fs)
        self._comp = [Field(grid, a + b, False, count, self._data[_slot(a, b)]) for a, b in PAIRS]

    @staticmethod
    def CanonicalIndices():
        return list(PAIRS)

    def __getitem__(self, ab) -> Field:
        a, b = ab
        return self._comp[_slot(a, b)]

    def Data(self):
        """The components, [9][count][nTheta * nPhi]."""
        return self._data

    def _same(self, o):
        if not isinstance(o, MatrixField) or o.grid is not self.grid or o.count != self.count:
            raise BadArgument(1, "matrix fields differ in grid or batch size")

    def _map(self, fn) -> "MatrixField":
        out = MatrixField(self.grid, self.count)
        for a, b in PAIRS:
            out[a, b].assign(fn(a, b), upper_index=a + b)
        return out

    # --- assignment and component-wise algebra ------------------------------
    def assign(self, o: "MatrixField") -> "MatrixField":
        self._same(o)
        for a, b in PAIRS:
            self[a, b].assign(o[a, b], upper_index=a + b)
        return self

    def __neg__(self):
        return self._map(lambda a, b: -self[a, b])

    def __add__(self, o):
        self._same(o)
        return self._map(lambda a, b: self[a, b] + o[a, b])

    def __sub__(self, o):
        self._same(o)
        return self._map(lambda a, b: self[a, b] - o[a, b])

    def __mul__(self, s):
        """By a complex scalar, or by a scalar field of upper index 0."""
        if isinstance(s, F.Expr) and s.N != 0:
            raise BadArgument(1, "matrix fields scale by scalar fields of upper index 0")
        return self._map(lambda a, b: self[a, b] * s)

    __rmul__ = __mul__

    def __iadd__(self, o):
        self._same(o)
        for a, b in PAIRS:
            self[a, b].assign(self[a, b] + o[a, b], upper_index=a + b)
        return self

    def __isub__(self, o):
        self._same(o)
        for a, b in PAIRS:
            self[a, b].assign(self[a, b] - o[a, b], upper_index=a + b)
        return self


def Transpose(A: MatrixField) -> MatrixField:
    """(A^T)_{alpha beta} = A_{beta alpha} (same upper index alpha + beta)."""
    return A._map(lambda a, b: A[b, a])


def Adjoint(A: MatrixField) -> MatrixField:
    """conj(A_{beta alpha}), the reference's complex adjoint
    (MatrixFieldExpressions.h:96-111); the conjugate of a component of
    upper index n has upper index -n, so A_{beta alpha} enters with index
    -(alpha + beta) and leaves with alpha + beta."""
    return A._map(lambda a, b: F.conj(A[b, a], upper_index=a + b))


def Action(A: MatrixField, u: VectorField) -> VectorField:
    """(A u)_alpha = -A_{alpha,-1} u_{+1} + A_{alpha,0} u_0 - A_{alpha,+1} u_{-1},
    one fused kernel per component."""
    if u.grid is not A.grid or u.count != A.count:
        raise BadArgument(1, "matrix and vector fields differ in grid or batch size")
    out = VectorField(A.grid, A.count)
    for a in CANONICAL_INDICES:
        expr = A[a, 0] * u[0] - A[a, -1] * u[1] - A[a, 1] * u[-1]
        out[a].assign(expr, upper_index=a)
    return out


def Multiply(A: MatrixField, B: MatrixField) -> MatrixField:
    """(A B)_{alpha beta} = -A_{alpha,+1} B_{-1,beta} + A_{alpha,0} B_{0,beta}
    - A_{alpha,-1} B_{+1,beta}, one fused kernel per component."""
    A._same(B)
    return A._map(lambda a, b: A[a, 0] * B[0, b] - A[a, 1] * B[-1, b] - A[a, -1] * B[1, b])


def Trace(A: MatrixField) -> Field:
    """g^{alpha beta} A_{alpha beta} = -A_{-1,+1} + A_{00} - A_{+1,-1}, a scalar
    field of upper index 0, in one fused kernel."""
    return (A[0, 0] - A[-1, 1] - A[1, -1]).evaluate(upper_index=0)


def Determinant(A: MatrixField) -> Field:
    """The cofactor expansion of MatrixFieldDeterminant's complex branch
    (MatrixFieldExpressions.h:359-369), a scalar field of upper index 0, in
    one fused kernel over the nine components."""
    e = (-A[-1, -1] * (A[0, 0] * A[1, 1] - A[0, 1] * A[1, 0])
         + A[-1, 0] * (A[0, -1] * A[1, 1] - A[0, 1] * A[1, -1])
         - A[-1, 1] * (A[0, -1] * A[1, 0] - A[0, 0] * A[1, -1]))
    return e.evaluate(upper_index=0)


def Isotropic(grid, a, count: int = 1) -> MatrixField:
    """IsotropicMatrixField (IsotropicMatrixField.h:26-33): A_{alpha beta} =
    (-1)^alpha a for alpha + beta = 0, zero otherwise; ``a`` is a complex
    scalar or a scalar field of upper index 0."""
    A = MatrixField(grid, count)
    for al in CANONICAL_INDICES:
        s = -1 if al % 2 else 1
        if isinstance(a, F.Expr):
            A[al, -al].assign(a * s, upper_index=0)
        else:
            A[al, -al].assign(complex(a) * s, upper_index=0)
    return A


class MatrixExpansion:
    """The nine canonical-component expansions of a matrix field: component
    (alpha, beta) holds c^{alpha beta}_lm of upper index alpha + beta."""

    def __init__(self, grid, count: int = 1, lmax: int | None = None):
        self.grid, self.count = grid, int(count)
        self._comp = [Expansion(grid, a + b, False, count, lmax=lmax) for a, b in PAIRS]
        self.lmax = self._comp[0].lmax

    def __getitem__(self, ab) -> Expansion:
        a, b = ab
        return self._comp[_slot(a, b)]

    def from_field(self, A: MatrixField, precision: str = "fp64") -> "MatrixExpansion":
        if A.grid is not self.grid or A.count != self.count:
            raise BadArgument(1, "matrix field and expansion differ in grid or batch size")
        for a, b in PAIRS:
            self[a, b].from_field(A[a, b], precision)
        return self

    def to_field(self, A: MatrixField | None = None, precision: str = "fp64") -> MatrixField:
        if A is None:
            A = MatrixField(self.grid, self.count)
        elif A.grid is not self.grid or A.count != self.count:
            raise BadArgument(1, "matrix field and expansion differ in grid or batch size")
        for a, b in PAIRS:
            self[a, b].to_field(A[a, b], precision)
        return A

    @classmethod
    def of(cls, A: MatrixField, precision: str = "fp64", lmax: int | None = None):
        return cls(A.grid, A.count, lmax=lmax).from_field(A, precision)
