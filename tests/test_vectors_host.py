"""Host-side bookkeeping of the vector-field layer (no GPU needed)."""

from __future__ import annotations

import pytest


def test_canonical_indices_and_checks():
    import gshtrans_b200 as g
    from gshtrans_b200 import vectors as V

    assert V.CANONICAL_INDICES == (-1, 0, 1)
    assert list(V.VectorField.CanonicalIndices()) == [-1, 0, 1]
    assert list(V.VectorExpansion.CanonicalIndices()) == [-1, 0, 1]
    for a in (-1, 0, 1):
        assert V._check_alpha(a) == a + 1
    for a in (-2, 2, 5):
        with pytest.raises(g.BadArgument):
            V._check_alpha(a)
