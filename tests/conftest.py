"""Shared test configuration.

Tests marked ``gpu`` need a CUDA device and the in-tree libgsht_cuda.so; the
rest run on CPU only (oracle pinning, host logic, the C-ABI surface, and the
multi-process host paths over gloo).
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libgsht_cuda.so")


@pytest.fixture(autouse=True, scope="module")
def _release_device_memory():
    """After each test module, return the device memory its objects held
    (collected grids, torch's cached blocks), so that the large-table tests
    (lmax 2048 grids take up to ~180 GB) see the whole GPU whatever ran
    before them. No-op where CUDA was never initialised."""
    yield
    if "torch" not in sys.modules:
        return
    import gc

    import torch

    gc.collect()
    if torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.synchronize()
        torch.cuda.empty_cache()


def relerr(a, b) -> float:
    """Norm-wise relative error ||a - b||_2 / ||b||_2."""
    a = np.asarray(a)
    b = np.asarray(b)
    nb = np.linalg.norm(b.ravel())
    d = np.linalg.norm((a - b).ravel())
    return float(d / nb) if nb > 0 else float(d)


@pytest.fixture(scope="session")
def golden():
    return {
        name: np.load(os.path.join(GOLDEN, f"{name}.npz"))
        for name in ("nodes", "wigner", "transforms", "wigner_single", "lmax2048")
    }


@pytest.fixture(scope="session")
def restated():
    import oracle

    return oracle.Restated()


@pytest.fixture(scope="session")
def reference():
    import oracle

    if not oracle.Reference.available():
        pytest.skip("reference build oracle/_ref is absent (built only where the reference tree exists)")
    return oracle.Reference()


def golden_cases(tr):
    """Yields (index, L, lmax, n, is_real) for every transform fixture."""
    for i in range(int(tr["count"])):
        L, lmax, n, is_real = (int(v) for v in tr[f"c{i}_meta"])
        yield i, L, lmax, n, bool(is_real)
