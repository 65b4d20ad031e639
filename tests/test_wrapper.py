"""Host-side argument checks of the Python wrappers (hyperalignment_b200/hyperalignment_c.py).

The library reads nt x nv of X and Y, nv + 1 column pointers and len(indices) rows, and writes
len(indices) float64 values into the caller's data. The wrappers check those shapes and types
before any device work, so a mismatch raises ValueError instead of reaching the C library. The
reference's own arrays (golden fixtures) pass the checks: the device call is stubbed here and
must be reached.
"""

import numpy as np
import pytest

from hyperalignment_b200 import hyperalignment_c as H

from conftest import golden


class _Reached(Exception):
    pass


@pytest.fixture
def stub_device(monkeypatch):
    def fake_init():
        raise _Reached()
    monkeypatch.setattr(H, "_init", fake_init)


def _lists(flat, off):
    return [flat[off[s]:off[s + 1]] for s in range(len(off) - 1)]


def test_reference_arrays_pass_the_checks(stub_device):
    g = golden("small_sparse.npz")
    sls = _lists(g["idx"], g["off"])
    ws = _lists(g["weights"], g["off"])
    data = np.zeros(g["indices"].size)
    with pytest.raises(_Reached):
        H.searchlight_procrustes(g["X"], g["Y"], sls, None, 0.0)
    with pytest.raises(_Reached):
        H.searchlight_procrustes_csc(g["X"], g["Y"], sls, g["indptr"], g["indices"], data, weights=ws)
    with pytest.raises(_Reached):
        H.searchlight_ridge_csc(g["X"], g["Y"], sls, g["indptr"], g["indices"], data, 1.0, weights=[g["weights"]])
    with pytest.raises(_Reached):
        H.searchlight_ridge_grid(g["X"], g["Y"], sls, g["indptr"], g["indices"], data, [1.0], [5],
                                 [np.arange(40)], [np.arange(5)])


@pytest.mark.parametrize("case", ["xy_shape", "indptr_len", "indptr_end", "data_dtype", "data_len",
                                  "data_readonly", "weights_len"])
def test_mismatches_raise_before_the_device(stub_device, case):
    g = golden("small_sparse.npz")
    X, Y = g["X"], g["Y"]
    sls = _lists(g["idx"], g["off"])
    indptr, indices = g["indptr"], g["indices"]
    data = np.zeros(indices.size)
    ws = [g["weights"]]
    if case == "xy_shape":
        Y = Y[:, :-1]
    elif case == "indptr_len":
        indptr = indptr[:-1]
    elif case == "indptr_end":
        indices = indices[:-1]
        data = np.zeros(indices.size)
    elif case == "data_dtype":
        data = np.zeros(indices.size, dtype=np.float32)
    elif case == "data_len":
        data = np.zeros(indices.size - 1)
    elif case == "data_readonly":
        data.flags.writeable = False
    elif case == "weights_len":
        ws = [g["weights"][:-1]]
    with pytest.raises(ValueError):
        H.searchlight_procrustes_csc(X, Y, sls, indptr, indices, data, weights=ws)
    with pytest.raises(ValueError):
        H.searchlight_ridge_csc(X, Y, sls, indptr, indices, data, 1.0, weights=ws)


def test_dense_shape_mismatch_raises(stub_device):
    X = np.zeros((10, 6))
    with pytest.raises(ValueError):
        H.searchlight_procrustes(X, np.zeros((10, 5)), [np.arange(3)], None, 0.0)
    with pytest.raises(ValueError):
        H.searchlight_procrustes(X, X, [np.arange(3)], None, 0.0, backend="cuda")
    with pytest.raises(ValueError):  # one distance short
        H.searchlight_procrustes(X, X, [np.arange(3)], [np.ones(2)], 2.0)
    with pytest.raises(ValueError):
        H.searchlight_weights([np.arange(3)], [np.ones(2)], 2.0)
