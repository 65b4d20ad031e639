"""C ABI checks that need no GPU: the library loads, exports every declared symbol,
and its host-only logic (argument checks, weights) matches the reference."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from hyperalignment_b200 import _lib as L

HEADER = os.path.join(ROOT, "include", "hyperalignment_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:int|void|bool|int64_t)\s+\**\s*(ha_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    # the reference wrapper binds these (hyperalignment_c.py:44-91)
    for n in ["ha_searchlight_procrustes_dense", "ha_set_num_threads", "ha_get_num_threads"]:
        assert n in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(hlib):
    missing = [n for n in declared_functions() if not hasattr(hlib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert sorted(L.SIGNATURES) == declared_functions()


def test_dense_rejects_non_b200_backend(hlib):
    # no CPU fallback: backends 0-3 belong to the reference library
    z = np.zeros(4)
    idx = np.zeros(1, dtype=np.int32)
    off = np.array([0, 1], dtype=np.int32)
    for backend in (0, 1, 2, 3, 5):
        rc = hlib.ha_searchlight_procrustes_dense(L.dptr(z), L.dptr(z), 2, 2, L.iptr(idx), L.iptr(off), None, 1,
                                                  1.0, L.dptr(z), True, False, backend, True)
        assert rc == L.ERROR_ARG


def test_weights_bit_exact_vs_reference(hlib):
    g = golden("small_sparse.npz")
    out = np.empty(g["idx"].size)
    rc = hlib.ha_searchlight_weights_b200(L.iptr(g["idx"]), L.iptr(g["off"]), L.dptr(g["dists"]),
                                          g["off"].size - 1, float(g["radius"]), g["X"].shape[1], L.dptr(out))
    assert rc == 0
    np.testing.assert_array_equal(out, g["weights"])
    out_u = np.empty(g["idx"].size)
    assert hlib.ha_searchlight_weights_b200(L.iptr(g["idx"]), L.iptr(g["off"]), None, g["off"].size - 1, 0.0,
                                            g["X"].shape[1], L.dptr(out_u)) == 0
    sums = np.zeros(g["X"].shape[1])
    np.add.at(sums, g["idx"], out_u)
    np.testing.assert_allclose(sums[sums > 0], 1.0, atol=1e-12)


@pytest.mark.parametrize("case", ["out_of_range", "duplicate", "empty", "bad_first_offset"])
def test_argument_errors(hlib, case):
    idx = np.array([0, 1, 2, 2, 3], dtype=np.int32)
    off = np.array([0, 3, 5], dtype=np.int32)
    nv = 4
    if case == "out_of_range":
        idx = np.array([0, 1, 9, 2, 3], dtype=np.int32)
    elif case == "duplicate":
        idx = np.array([0, 1, 1, 2, 3], dtype=np.int32)
    elif case == "empty":
        off = np.array([0, 0, 5], dtype=np.int32)
    elif case == "bad_first_offset":
        off = np.array([1, 3, 5], dtype=np.int32)
    out = np.empty(idx.size)
    rc = hlib.ha_searchlight_weights_b200(L.iptr(idx), L.iptr(off), None, 2, 0.0, nv, L.dptr(out))
    assert rc == L.ERROR_ARG


def test_init_reports_missing_gpu(hlib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    assert hlib.ha_b200_init() == L.ERROR_INTERNAL
    assert not hlib.ha_b200_available()
