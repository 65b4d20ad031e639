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


@pytest.mark.parametrize("pre,args,mask", [("cv", (500, 1, 5, 10, 10, 5), False), ("cvm", (150, 2, 3, 7, 4, 9), True)])
def test_ensemble_indices_c_abi_bit_exact(hlib, pre, args, mask):
    # host-only entry: the same draws as the reference's ha_ensemble_indices
    from hyperalignment_b200 import hyperalignment_c as H
    g = golden("grid.npz")
    tr, te = H.ensemble_indices(*args, mask=g["cvm_mask"] if mask else None)
    sizes = g[pre + "_test_sizes"]
    rte = np.split(g[pre + "_test"], np.cumsum(sizes)[:-1])
    for a, b in zip(tr, g[pre + "_train"]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(te, rte):
        np.testing.assert_array_equal(a, b)


def test_ensemble_indices_argument_errors(hlib):
    buf = np.zeros(100, dtype=np.int32)
    sz = np.zeros(4, dtype=np.int32)
    # blocksize 0 (the reference divides by it), and a single fold that leaves no training rows
    assert hlib.ha_ensemble_indices_b200(20, 1, 2, 0, 1, 1, None, L.iptr(buf), L.iptr(buf), L.iptr(sz)) == L.ERROR_ARG
    assert hlib.ha_ensemble_indices_b200(20, 1, 1, 5, 2, 1, None, L.iptr(buf), L.iptr(buf), L.iptr(sz)) == L.ERROR_ARG


def test_ridge_grid_argument_errors(hlib):
    # checked on the host before any device work: negative PC counts, a repeated test row,
    # a training row outside [0, nt), an empty training list
    X = np.zeros((10, 4))
    sls = [np.array([0, 1], dtype=np.int32), np.array([2, 3], dtype=np.int32)]
    indptr = np.array([0, 2, 4, 6, 8], dtype=np.int32)
    indices = np.array([0, 1, 0, 1, 2, 3, 2, 3], dtype=np.int32)
    data = np.zeros(8)
    ok_tr, ok_te = [np.arange(10)], [np.arange(3)]
    bad = [
        ([1.0], [-1], ok_tr, ok_te),
        ([1.0], [2], ok_tr, [np.array([1, 1])]),
        ([1.0], [2], [np.array([0, 10])], ok_te),
        ([1.0], [2], [np.zeros(0)], ok_te),
        ([float("nan")], [2], ok_tr, ok_te),
    ]
    idx = np.concatenate(sls)
    off = np.array([0, 2, 4], dtype=np.int32)
    best = np.zeros(2, dtype=np.int32)
    for alphas, npcs, tr, te in bad:
        al = np.asarray(alphas, dtype=np.float64)
        pc = np.asarray(npcs, dtype=np.int32)
        trl, tel = L.IndexLists(tr), L.IndexLists(te)
        rc = hlib.ha_searchlight_ridge_grid_b200(
            L.dptr(X), L.dptr(X), 10, 4, L.iptr(idx), L.iptr(off), 2, None, L.iptr(indptr), L.iptr(indices), 8,
            L.dptr(data), L.dptr(al), al.size, L.iptr(pc), pc.size, trl.ptrs, tel.ptrs, L.iptr(trl.sizes),
            L.iptr(tel.sizes), 1, L.iptr(best), None, True)
        assert rc == L.ERROR_ARG


def test_mlp_parameter_count_and_argument_errors(hlib):
    # 65 -> 128 -> 128 -> C with biases; C outside 1..64 is rejected
    for C in (1, 40, 64):
        assert hlib.ha_b200_mlp_param_count(C) == 65 * 128 + 128 + 128 * 128 + 128 + 128 * C + C
    assert hlib.ha_b200_mlp_param_count(0) == -1 and hlib.ha_b200_mlp_param_count(65) == -1
    # checked before any device work: missing buffers, empty sets, non-positive learning rate
    buf = ctypes.c_void_p(1)
    assert hlib.ha_b200_mlp_train(None, 40, buf, buf, 10, 1, 8, 1e-3, 0, None) == L.ERROR_ARG
    assert hlib.ha_b200_mlp_train(buf, 40, buf, buf, 0, 1, 8, 1e-3, 0, None) == L.ERROR_ARG
    assert hlib.ha_b200_mlp_train(buf, 40, buf, buf, 10, 1, 8, 0.0, 0, None) == L.ERROR_ARG
    assert hlib.ha_b200_mlp_grad(buf, 40, buf, buf, 0, buf, None) == L.ERROR_ARG
    assert hlib.ha_b200_mlp_infer(buf, 40, buf, -1, buf, buf, None) == L.ERROR_ARG
    assert hlib.ha_b200_mlp_init(None, 40, 0) == L.ERROR_ARG


def test_aligned_correlation_argument_errors(hlib):
    # checked on the host before any device work; the non-null pointers here are never read
    f = hlib.ha_b200_aligned_correlation_device
    p = 4096
    assert f(None, p, 10, 4, None, None, None, 0, p, None, None) == L.ERROR_ARG   # no X
    assert f(p, p, 10, 4, None, None, None, 0, None, None, None) == L.ERROR_ARG   # no output
    assert f(p, p, 0, 4, None, None, None, 0, p, None, None) == L.ERROR_ARG       # nt < 1
    assert f(p, p, 10, 0, None, None, None, 0, p, None, None) == L.ERROR_ARG      # nv < 1
    assert f(p, p, 10, 4, None, p, p, 8, p, None, None) == L.ERROR_ARG            # values without indptr
    assert f(p, p, 10, 4, p, None, p, 8, p, None, None) == L.ERROR_ARG            # values without rows
    assert f(p, p, 10, 4, p, p, p, -1, p, None, None) == L.ERROR_ARG              # negative nnz


@pytest.mark.parametrize("args,mask_seed", [
    ((300, 3, 4, 8, 0, 11), None), ((97, 2, 3, 5, 2, 0), None), ((64, 1, 2, 16, 4, 123456789), None),
    ((500, 1, 5, 10, 10, 5), None), ((500, 4, 5, 10, 10, 2**63 + 7), None), ((41, 2, 7, 1, 0, 3), None),
    ((200, 2, 4, 6, 3, 17), 1), ((150, 1, 5, 10, 10, 99), 2),
])
def test_ensemble_indices_c_abi_vs_live_reference(hlib, args, mask_seed):
    """The library's host split generator against the compiled reference's ha_ensemble_indices
    (csrc/ha_ensemble.c:58-249), draw for draw, over fold counts, block and buffer sizes,
    several permutations, 64-bit seeds and masks."""
    from oracle import ref_lib as R
    if not R.available():
        pytest.skip("compiled reference not built (make -C oracle)")
    from hyperalignment_b200 import hyperalignment_c as H
    mask = None
    if mask_seed is not None:
        mask = np.random.default_rng(mask_seed).random(args[0]) < 0.8
    tr, te = H.ensemble_indices(*args, mask=mask)
    rtr, rte = R.ensemble_indices(*args, mask=mask)
    assert len(tr) == len(rtr) == len(te) == len(rte)
    for a, b in zip(tr + te, rtr + rte):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("seed,uniform", [(0, False), (1, True), (2, False), (3, True)])
def test_weights_c_abi_vs_live_reference(hlib, seed, uniform):
    """The library's host weights (the rule of csrc/ha_searchlight.c:970-1001 and :36-92) against
    the compiled reference's ha_searchlight_weights, bit for bit, on ragged k-NN searchlights with
    distance weights and uniform ones."""
    from oracle import ref_lib as R
    if not R.available():
        pytest.skip("compiled reference not built (make -C oracle)")
    from hyperalignment_b200 import hyperalignment_c as H
    from hyperalignment_b200 import workloads as W
    s = W.small_case(seed=seed, nv=642, nt=8, lo=5, hi=70).sls
    sls = [s.indices[s.offsets[q]:s.offsets[q + 1]] for q in range(s.count)]
    ds = None if uniform else [s.dists[s.offsets[q]:s.offsets[q + 1]] for q in range(s.count)]
    ours = H.searchlight_weights(sls, ds, None if uniform else s.radius, 642)
    ref = R.searchlight_weights(s.indices, s.offsets, None if uniform else s.dists, 0.0 if uniform else s.radius)
    assert np.array_equal(ours, ref)


def test_grid_precision_argument_errors(hlib):
    # a plan is needed, and only 32 or 64 bits are accepted (checked before any device work)
    for bits in (32, 64, 16, 0):
        assert hlib.ha_b200_plan_set_grid_precision(None, bits) == L.ERROR_ARG
