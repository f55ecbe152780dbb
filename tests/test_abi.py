"""The C-ABI library loads and exports every symbol include/gsht.h declares;
host-side validation that needs no GPU."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from conftest import ROOT

import oracle


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "gsht.h")).read()
    return sorted(set(re.findall(r"\b(gsht_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import gshtrans_b200 as g

    syms = declared_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(g.library, s), s


def test_coefficient_sizes_match_reference_layout():
    import gshtrans_b200 as g

    for lmax in (0, 1, 5, 64, 1024):
        for n in range(-min(lmax, 3), min(lmax, 3) + 1):
            assert g.coefficient_size(lmax, n, False) == oracle.size_all(lmax, n)
            assert g.coefficient_size(lmax, n, True) == oracle.size_nonneg(lmax, n)
    with pytest.raises(g.BadArgument):
        g.coefficient_size(2, 3, False)


def test_grid_create_rejects_bad_arguments_before_touching_a_device():
    import gshtrans_b200 as g

    lib = g.library
    h = ctypes.c_void_p()
    assert lib.gsht_grid_create(0, 0, 0, 0, 1, ctypes.byref(h)) == 1
    assert b"lmax" in lib.gsht_last_error()
    assert lib.gsht_grid_create(8, 9, 0, 0, 1, ctypes.byref(h)) == 1
    assert lib.gsht_grid_create(8, 2, 2, 0, 1, ctypes.byref(h)) == 1
    assert lib.gsht_grid_create(8, 2, 0, 0, 64, ctypes.byref(h)) == 1
    assert lib.gsht_grid_create(8, 2, 0, 0, 1, None) == 1


def test_no_device_is_reported_not_faked():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import gshtrans_b200 as g

    with pytest.raises(g.GSHTError) as e:
        g.GaussLegendreGrid(8, 2)
    assert e.value.status == 6


def test_wigner_compute_validates_and_sizes_without_a_device():
    import gshtrans_b200 as g

    lib = g.library
    cnt = ctypes.c_long()
    th = (ctypes.c_double * 3)(0.1, 0.2, 0.3)
    # Count-only query: Wigner<double, Ortho, All, All>(20, 7, 3) at 3 angles.
    assert lib.gsht_wigner_compute(20, 7, 3, 0, 0, 0, 0, th, 3, None, ctypes.byref(cnt)) == 0
    want = 0
    for n in range(-3, 4):
        want += 3 * sum(2 * min(l, 7) + 1 for l in range(abs(n), 21))
    assert cnt.value == want
    with pytest.raises(g.BadArgument):
        g.wigner(10, 10, 11, 0.5)          # nMax > lMax
    with pytest.raises(g.BadArgument):
        g.wigner(10, -1, 1, 0.5)           # negative mMax
    with pytest.raises(g.BadArgument):
        g.wigner(10, 10, 1, 0.5, mrange=2)  # MRange must be All or NonNegative


def test_plan_batch_validates_without_a_device():
    import gshtrans_b200 as g

    d = g._FieldDesc(64, 0, 0, 1, 1, 1)
    arr = (g._FieldDesc * 1)(d)
    h = ctypes.c_void_p()
    assert g.library.gsht_plan_batch(arr, 0, 1, 1, ctypes.byref(h)) == 1       # no fields
    bad = (g._FieldDesc * 1)(g._FieldDesc(0, 0, 0, 1, 1, 1))
    assert g.library.gsht_plan_batch(bad, 1, 1, 1, ctypes.byref(h)) == 1       # lmax 0
    bad = (g._FieldDesc * 1)(g._FieldDesc(8, 9, 0, 1, 1, 1))
    assert g.library.gsht_plan_batch(bad, 1, 1, 1, ctypes.byref(h)) == 1       # |n| > lmax
    bad = (g._FieldDesc * 1)(g._FieldDesc(8, 0, 0, None, 1, 1))
    assert g.library.gsht_plan_batch(bad, 1, 1, 1, ctypes.byref(h)) == 1       # NULL buffer
    assert g.library.gsht_plan_batch(arr, 1, 7, 1, ctypes.byref(h)) == 5       # precision
    assert g.library.gsht_plan_batch(arr, 1, 1, 1, ctypes.byref(h)) == 6       # no device
    assert g.library.gsht_batch_execute(None, 0, None) == 1


def test_python_constants_match_the_header():
    # The Python mirror's precision and form constants are the C ABI's.
    import gshtrans_b200 as g

    text = open(os.path.join(ROOT, "include", "gsht.h")).read()
    values = {k: int(v) for k, v in re.findall(r"\b(GSHT_[A-Z0-9_]+)\s*=\s*(\d+)", text)}
    for name in ("FP64", "BF16X3", "OZAKI", "RECURRENCE", "OZAKI4"):
        assert getattr(g, name) == values[f"GSHT_{name}"], name
    forms = {"FP64": "GSHT_FORM_FP64", "BF16X3": "GSHT_FORM_BF16X3", "OZAKI": "GSHT_FORM_OZAKI",
             "RECURRENCE": "GSHT_FORM_RECURRENCE", "OZAKI4": "GSHT_FORM_OZAKI"}
    for name, form in forms.items():
        assert g._FORM_BIT[getattr(g, name)] == values[form], name
    for name, code in (("All", "GSHT_RANGE_ALL"), ("NonNegative", "GSHT_RANGE_NONNEGATIVE"),
                       ("Single", "GSHT_RANGE_SINGLE")):
        assert getattr(g, name) == values[code], name


def test_stage_profile_without_calls():
    # No transform inside the block: every stage reads zero (no device needed).
    import gshtrans_b200 as g

    with g.StageProfile() as p:
        pass
    assert tuple(p.stages) == g.STAGES
    assert all(v == (0.0, 0) for v in p.stages.values())


def test_trace_read_rejects_bad_arguments_without_a_device():
    import gshtrans_b200 as gsht

    with pytest.raises(gsht.BadArgument):
        gsht.TensorCoreTrace.read("fp64", 0)
    with pytest.raises(gsht.BadArgument):
        gsht.TensorCoreTrace.read("bf16x3", 2)
