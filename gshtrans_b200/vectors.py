"""Vector fields in canonical components, and their expansions.

Python mirror of the reference's (header-disabled) vector-field layer:
``CanonicalVector`` indices alpha = -1, 0, +1 (src/VectorField/CanonicalVector.h
:13-22), component access and compound operators of ``VectorFieldBase``
(VectorFieldBase.h), the component-wise unary and scalar / scalar-field
forms and the pointwise ``InnerProduct`` and ``DualityProduct``
(VectorFieldOverloads.h:26-300). The canonical component alpha of a vector
field is a ``CanonicalComponentField`` of upper index alpha, so each one
transforms with the grid's table of n = alpha; ``VectorExpansion`` holds the
three coefficient sets and runs the three transforms (each batched over
``count`` fields) on the caller's stream.

Complex-valued fields carry the canonical components. The reference's
real-valued branch (a real vector field in the real basis u_{-1}, u_0, u_{+1})
is ``RealVectorField``, with the two conversions of
VectorFieldRealToComplex.h:66-72 (``complexify``) and
VectorFieldComplexToReal.h:62-69 (``realify``); its components have no
transform of their own (transform the complexified field).

The three components live in one CUDA tensor [3][count][nTheta * nPhi];
pointwise operations run the fused expression kernel once per component
(``gsht_field_eval``), the products once in total.
"""

from __future__ import annotations

from . import BadArgument
from . import fields as F
from .expansions import Expansion
from .fields import Field

CANONICAL_INDICES = (-1, 0, 1)


def _check_alpha(alpha: int) -> int:
    if alpha not in CANONICAL_INDICES:
        raise BadArgument(1, f"canonical index {alpha} not in -1, 0, +1")
    return alpha + 1


class VectorField:
    """VectorField<Grid, ComplexValued> on the GPU: components u_alpha."""

    def __init__(self, grid, count: int = 1, data=None):
        import torch

        self.grid, self.count = grid, int(count)
        fs = grid.FieldSize()
        if grid.MaxUpperIndex() < 1 or grid.MinUpperIndex() > -1:
            raise BadArgument(1, "vector fields need a grid with upper indices -1..1")
        if data is None:
            self._data = torch.zeros((3, count, fs), dtype=torch.complex128, device="cuda")
        else:
            if data.dtype != torch.complex128 or data.numel() != 3 * count * fs or not data.is_cuda:
                raise BadArgument(1, "data must be a complex128 CUDA tensor of 3 x count fields")
            self._data = data.contiguous().view(3, count, fs)
        self._comp = [Field(grid, a, False, count, self._data[a + 1]) for a in CANONICAL_INDICES]

    # --- access (VectorFieldBase.h: operator[](alpha), CanonicalIndices) -----
    @staticmethod
    def CanonicalIndices():
        return range(-1, 2)

    def __getitem__(self, alpha: int) -> Field:
        return self._comp[_check_alpha(alpha)]

    def Data(self):
        """The components, [3][count][nTheta * nPhi] (alpha = -1, 0, +1)."""
        return self._data

    def _same(self, o: "VectorField"):
        if not isinstance(o, VectorField) or o.grid is not self.grid or o.count != self.count:
            raise BadArgument(1, "vector fields differ in grid or batch size")

    # --- assignment and compound operators ----------------------------------
    def assign(self, o: "VectorField") -> "VectorField":
        self._same(o)
        for a in CANONICAL_INDICES:
            self[a].assign(o[a])
        return self

    def __iadd__(self, o):
        self._same(o)
        for a in CANONICAL_INDICES:
            self[a].assign(self[a] + o[a])
        return self

    def __isub__(self, o):
        self._same(o)
        for a in CANONICAL_INDICES:
            self[a].assign(self[a] - o[a])
        return self

    def __imul__(self, s):
        """By a scalar or by a scalar field (upper index 0)."""
        self._scale_check(s)
        for a in CANONICAL_INDICES:
            self[a].assign(self[a] * s, upper_index=a)
        return self

    def __itruediv__(self, s):
        self._scale_check(s)
        for a in CANONICAL_INDICES:
            self[a].assign(self[a] / s, upper_index=a)
        return self

    def _scale_check(self, s):
        if isinstance(s, F.Expr):
            if s.N != 0:
                raise BadArgument(1, "vector fields scale by scalar fields of upper index 0")
            g, count = s._geometry()
            if g is not self.grid or count != self.count:
                raise BadArgument(1, "scalar field differs in grid or batch size")

    # --- component-wise forms (VectorFieldOverloads.h:26-173) ---------------
    def _map(self, fn) -> "VectorField":
        out = VectorField(self.grid, self.count)
        for a in CANONICAL_INDICES:
            out[a].assign(fn(a), upper_index=a)
        return out

    def __neg__(self):
        return self._map(lambda a: -self[a])

    def __add__(self, o):
        self._same(o)
        return self._map(lambda a: self[a] + o[a])

    def __sub__(self, o):
        self._same(o)
        return self._map(lambda a: self[a] - o[a])

    def __mul__(self, s):
        self._scale_check(s)
        return self._map(lambda a: self[a] * s)

    __rmul__ = __mul__

    def __truediv__(self, s):
        self._scale_check(s)
        return self._map(lambda a: self[a] / s)


def conj(u: VectorField) -> VectorField:
    """Component-wise complex conjugate (VectorFieldOverloads.h:76-87). As for
    scalar fields the reference keeps each component's index alpha."""
    return u._map(lambda a: F.conj(u[a]))


def InnerProduct(u: VectorField, v: VectorField) -> Field:
    """sum_alpha conj(u_alpha) v_alpha, a scalar field of upper index 0
    (VectorFieldOverloads.h:240-252), in one fused kernel over the six
    components."""
    u._same(v)
    expr = None
    for a in CANONICAL_INDICES:
        term = F.conj(u[a], upper_index=-a) * v[a]
        expr = term if expr is None else expr + term
    return expr.evaluate(upper_index=0)


def DualityProduct(u: VectorField, v: VectorField) -> Field:
    """-u_{-1} v_{+1} + u_0 v_0 - u_{+1} v_{-1}, a scalar field of upper index
    0 (VectorFieldOverloads.h:276-288), in one fused kernel."""
    u._same(v)
    expr = u[0] * v[0] - u[-1] * v[1] - u[1] * v[-1]
    return expr.evaluate(upper_index=0)


class VectorExpansion:
    """The three canonical-component expansions of a vector field: component
    alpha holds c^alpha_lm for degrees max(|alpha|, 0)..lmax."""

    def __init__(self, grid, count: int = 1, lmax: int | None = None):
        self.grid, self.count = grid, int(count)
        self._comp = [Expansion(grid, a, False, count, lmax=lmax) for a in CANONICAL_INDICES]
        self.lmax = self._comp[0].lmax

    @staticmethod
    def CanonicalIndices():
        return range(-1, 2)

    def __getitem__(self, alpha: int) -> Expansion:
        return self._comp[_check_alpha(alpha)]

    def from_field(self, u: VectorField, precision: str = "fp64") -> "VectorExpansion":
        """Forward transforms of the three components (each replaces the
        component's coefficients)."""
        if u.grid is not self.grid or u.count != self.count:
            raise BadArgument(1, "vector field and expansion differ in grid or batch size")
        for a in CANONICAL_INDICES:
            self[a].from_field(u[a], precision)
        return self

    def to_field(self, u: VectorField | None = None, precision: str = "fp64") -> VectorField:
        """Inverse transforms of the three components into ``u`` (new if None)."""
        if u is None:
            u = VectorField(self.grid, self.count)
        elif u.grid is not self.grid or u.count != self.count:
            raise BadArgument(1, "vector field and expansion differ in grid or batch size")
        for a in CANONICAL_INDICES:
            self[a].to_field(u[a], precision)
        return u

    @classmethod
    def of(cls, u: VectorField, precision: str = "fp64", lmax: int | None = None):
        return cls(u.grid, u.count, lmax=lmax).from_field(u, precision)


class RealVectorField:
    """VectorField<Grid, RealValued> on the GPU: three real components in the
    reference's real basis, one CUDA tensor [3][count][nTheta * nPhi]
    (alpha = -1, 0, +1)."""

    def __init__(self, grid, count: int = 1, data=None):
        import torch

        self.grid, self.count = grid, int(count)
        fs = grid.FieldSize()
        if data is None:
            self._data = torch.zeros((3, count, fs), dtype=torch.float64, device="cuda")
        else:
            if data.dtype != torch.float64 or data.numel() != 3 * count * fs or not data.is_cuda:
                raise BadArgument(1, "data must be a float64 CUDA tensor of 3 x count fields")
            self._data = data.contiguous().view(3, count, fs)
        self._comp = [Field(grid, 0, True, count, self._data[a + 1]) for a in CANONICAL_INDICES]

    @staticmethod
    def CanonicalIndices():
        return range(-1, 2)

    def __getitem__(self, alpha: int) -> Field:
        return self._comp[_check_alpha(alpha)]

    def Data(self):
        return self._data

    def _same(self, o):
        if not isinstance(o, RealVectorField) or o.grid is not self.grid or o.count != self.count:
            raise BadArgument(1, "real vector fields differ in grid or batch size")

    def _map(self, fn) -> "RealVectorField":
        out = RealVectorField(self.grid, self.count)
        for a in CANONICAL_INDICES:
            out[a].assign(fn(a), upper_index=0)
        return out

    def assign(self, o: "RealVectorField") -> "RealVectorField":
        self._same(o)
        for a in CANONICAL_INDICES:
            self[a].assign(o[a], upper_index=0)
        return self

    def __neg__(self):
        return self._map(lambda a: -self[a])

    def __add__(self, o):
        self._same(o)
        return self._map(lambda a: self[a] + o[a])

    def __sub__(self, o):
        self._same(o)
        return self._map(lambda a: self[a] - o[a])

    def __mul__(self, s):
        """By a real scalar or by a real scalar field."""
        if isinstance(s, complex) or (isinstance(s, F.Expr) and not s.is_real):
            raise BadArgument(1, "real vector fields scale by real scalars or real fields")
        return self._map(lambda a: self[a] * s)

    __rmul__ = __mul__


def complexify(u: RealVectorField) -> VectorField:
    """VectorFieldRealToComplex (VectorFieldRealToComplex.h:66-72): canonical
    components c_0 = u_0, c_alpha = alpha u_{+1} + i u_{-1} (alpha = +-1), one
    fused kernel per component."""
    out = VectorField(u.grid, u.count)
    out[0].assign(u[0] + 0j, upper_index=0)
    for a in (-1, 1):
        # (real field + 0j) is the field as a complex value; the operations
        # then stay within one value type, as the reference requires.
        out[a].assign(a * (u[1] + 0j) + 1j * (u[-1] + 0j), upper_index=a)
    return out


def realify(v: VectorField) -> RealVectorField:
    """VectorFieldComplexToReal (VectorFieldComplexToReal.h:62-69): with
    w_alpha = (v_alpha + (-1)^alpha conj(v_{-alpha})) / 2, the real components
    are Im w_alpha for alpha < 0 and Re w_alpha otherwise."""
    out = RealVectorField(v.grid, v.count)
    for a in CANONICAL_INDICES:
        sgn = -1.0 if a % 2 else 1.0
        w = 0.5 * (v[a] + sgn * F.conj(v[-a], upper_index=a))
        out[a].assign(F.imag(w) if a < 0 else F.real(w), upper_index=0)
    return out


def RealInnerProduct(u: RealVectorField, v: RealVectorField) -> Field:
    """sum_alpha u_alpha v_alpha of two real vector fields (the reference's
    real-valued InnerProduct, VectorFieldOverloads.h:244-249), one fused kernel."""
    u._same(v)
    return (u[-1] * v[-1] + u[0] * v[0] + u[1] * v[1]).evaluate(upper_index=0)
