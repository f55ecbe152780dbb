"""Canonical-component expansions: coefficients wired to the transforms.

Python mirror of the reference's ``CanonicalComponentExpansion<N, Grid,
Value>`` (CanonicalComponentExpansion.h:36-105, CanonicalComponentExpansionBase
.h:14-160): the coefficients c_lm of one upper index N for degrees |N|..L of a
grid, in the packed order of the transforms (``GSHIndices<All>`` for complex
fields, ``GSHIndices<NonNegative>`` for real ones), always complex. The
reference declares the container but never connects it to the grid's
transforms; here ``from_field`` (forward transform) and ``to_field`` (inverse)
run them on the GPU, for one expansion or a batch of ``count`` of them.

Coefficients live in a CUDA tensor; element access by (l, m) goes through
``Index`` (Indexing.h:104-131) and copies one value to or from the host.
"""

from __future__ import annotations

from . import BadArgument, coefficient_size
from .fields import Field


class Expansion:
    """CanonicalComponentExpansion<N, Grid, RealValued|ComplexValued> on the GPU."""

    def __init__(self, grid, n: int, is_real: bool = False, count: int = 1, data=None,
                 lmax: int | None = None):
        import torch

        self.grid, self.N, self.is_real, self.count = grid, int(n), bool(is_real), int(count)
        self.lmax = grid.MaxDegree() if lmax is None else int(lmax)
        if abs(self.N) > self.lmax or self.lmax > grid.MaxDegree():
            raise BadArgument(1, f"no expansion of upper index {n} to degree {self.lmax} on this grid")
        size = coefficient_size(self.lmax, self.N, self.is_real)
        shape = (count, size) if count > 1 else (size,)
        if data is None:
            self._data = torch.zeros(shape, dtype=torch.complex128, device="cuda")
        else:
            if data.dtype != torch.complex128 or data.numel() != count * size or not data.is_cuda:
                raise BadArgument(1, "data must be a complex128 CUDA tensor of the expansion's size")
            self._data = data.contiguous().view(shape)

    # --- bookkeeping (GSHIndices, Indexing.h:72-156) -------------------------
    def UpperIndex(self) -> int:
        return self.N

    def MinDegree(self) -> int:
        return abs(self.N)

    def MaxDegree(self) -> int:
        return self.lmax

    def Degrees(self):
        return range(self.MinDegree(), self.lmax + 1)

    def Size(self) -> int:
        return coefficient_size(self.lmax, self.N, self.is_real)

    def Index(self, l: int, m: int) -> int:
        na = abs(self.N)
        if not (na <= l <= self.lmax) or abs(m) > l or (self.is_real and m < 0):
            raise BadArgument(1, f"(l, m) = ({l}, {m}) not in the expansion")
        if self.is_real:
            return l * (l + 1) // 2 - na * (na + 1) // 2 + m
        return l * l - na * na + l + m

    def Data(self):
        """The packed coefficients (a CUDA tensor)."""
        return self._data

    def __getitem__(self, lm):
        l, m = lm
        return complex(self._data[..., self.Index(l, m)].item()) if self.count == 1 else \
            self._data[:, self.Index(l, m)].cpu().numpy()

    def __setitem__(self, lm, value):
        l, m = lm
        self._data[..., self.Index(l, m)] = value

    # --- transforms ---------------------------------------------------------
    def from_field(self, field: Field, precision: str = "fp64") -> "Expansion":
        """Replaces the coefficients by the field's (the grid's forward
        transform, which adds into its output, runs on zeroed coefficients)."""
        self._check_field(field)
        self._data.zero_()
        if self.count == 1:
            self.grid.ForwardTransformation(self.lmax, self.N, field.Data(), self._data, precision)
        else:
            self.grid.forward_batch(self.lmax, self.N, field.Data(), self._data, precision)
        return self

    def to_field(self, field: Field | None = None, precision: str = "fp64") -> Field:
        """The field with these coefficients (inverse transform), written into
        ``field`` if given."""
        if field is None:
            field = Field(self.grid, self.N, self.is_real, self.count)
        self._check_field(field)
        if self.count == 1:
            self.grid.InverseTransformation(self.lmax, self.N, self._data, field.Data(), precision)
        else:
            self.grid.inverse_batch(self.lmax, self.N, self._data, field.Data(), precision)
        return field

    @classmethod
    def of(cls, field: Field, precision: str = "fp64", lmax: int | None = None) -> "Expansion":
        """The expansion of a field (the reference's converting constructor)."""
        e = cls(field.grid, field.N, field.is_real, field.count, lmax=lmax)
        return e.from_field(field, precision)

    def _check_field(self, field: Field):
        if field.grid is not self.grid or field.N != self.N or field.is_real != self.is_real \
                or field.count != self.count:
            raise BadArgument(1, "field and expansion differ in grid, upper index, kind or batch size")

    # --- assignment and compound operators (Base :77-160) --------------------
    def _same(self, o: "Expansion"):
        if not isinstance(o, Expansion) or o.N != self.N or o.lmax != self.lmax \
                or o.is_real != self.is_real or o.count != self.count:
            raise BadArgument(1, "expansions differ in upper index, degree, kind or batch size")

    def assign(self, o: "Expansion") -> "Expansion":
        self._same(o)
        self._data.copy_(o._data)
        return self

    def __iadd__(self, o):
        self._same(o)
        self._data += o._data
        return self

    def __isub__(self, o):
        self._same(o)
        self._data -= o._data
        return self

    def __imul__(self, s):
        self._data *= complex(s)
        return self

    def __itruediv__(self, s):
        self._data /= complex(s)
        return self
