"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference checkout and its compiled library
(``make -C oracle``):

    python tests/golden/make_golden.py

Outputs (small, seeded inputs stored alongside the outputs so the fixtures are
self-contained):
  small_dense.npz   searchlight Procrustes through the reference dense entry point
                    (ha_searchlight_procrustes_dense, cpu64 and cpu32), with and without
                    reflection / scaling
  small_sparse.npz  ha_sparse_init pattern, ha_searchlight_weights, sparse-API Procrustes
                    and ridge (ha_searchlight_procrustes, ha_searchlight_ridge) CSC data
  kat.npz           outputs of ha_procrustes / ha_ridge on the reference harness's
                    known-answer inputs (csrc/ha_test.c:234-366, splitmix64 data)
  grid.npz          ha_ensemble_indices splits (with and without a mask), ha_ridge_grid betas
                    (monotone and non-monotone PC counts, bootstrap rows) and ha_ensemble_ridge
                    outputs on seeded inputs
  python_ref.npz    the Python reference package (src/hyperalignment) on the same small
                    case: procrustes per searchlight and initialize_sparse_matrix
  pca_template.npz  searchlight_template(tpl_kind="pca") of the Python reference package on
                    four subjects sharing one latent time series plus 1% noise, so that every
                    searchlight's top singular subspace is separated from the rest

    python tests/golden/make_golden.py [name ...]   # only the named fixtures (file stems)
"""

from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hyperalignment_b200 import workloads as W  # noqa: E402
from oracle import ha_oracle as O  # noqa: E402
from oracle import ref_lib as R  # noqa: E402

def _reference_dir():
    """HA_REFERENCE_DIR, else a checkout named "reference" beside this repository."""
    for cand in (os.environ.get("HA_REFERENCE_DIR"), os.path.join(os.path.dirname(ROOT), "reference")):
        if cand and os.path.isdir(os.path.join(cand, "src", "hyperalignment")):
            return os.path.abspath(cand)
    raise SystemExit("make_golden.py: set HA_REFERENCE_DIR to the neurolabusc/hyperalignment checkout")


REF_DIR = _reference_dir()


def small_inputs(seed=0):
    w = W.small_case(seed=seed)
    return w


def make_small_dense():
    w = small_inputs(0)
    s = w.sls
    out = dict(X=w.X, Y=w.Y, idx=s.indices, off=s.offsets, dists=s.dists, radius=np.float64(s.radius))
    R.set_threads(1)
    out["T_cpu64"] = R.procrustes_dense(w.X, w.Y, s.indices, s.offsets, s.dists, s.radius, True, False, 0)
    out["T_cpu32"] = R.procrustes_dense(w.X, w.Y, s.indices, s.offsets, s.dists, s.radius, True, False, 1)
    out["T_cpu64_noref_scal"] = R.procrustes_dense(w.X, w.Y, s.indices, s.offsets, s.dists, s.radius, False, True, 0)
    out["T_cpu64_uniform"] = R.procrustes_dense(w.X, w.Y, s.indices, s.offsets, None, 0.0, True, False, 0)
    np.savez_compressed(os.path.join(HERE, "small_dense.npz"), **out)


def make_small_sparse():
    w = small_inputs(1)
    s = w.sls
    indptr, indices = R.sparse_init(s.indices, s.offsets, w.nv)
    weights = R.searchlight_weights(s.indices, s.offsets, s.dists, s.radius)
    R.set_threads(1)
    data = R.searchlight_procrustes_csc(w.X, w.Y, s.indices, s.offsets, indptr, indices, weights, True, False, 0)
    data_unw = R.searchlight_procrustes_csc(w.X, w.Y, s.indices, s.offsets, indptr, indices, None, True, True, 0)
    data_ridge = R.searchlight_ridge_csc(w.X, w.Y, s.indices, s.offsets, indptr, indices, 1.0, weights)
    toy_idx = np.array([0, 1, 2, 1, 2, 3, 4], dtype=np.int32)  # csrc/ha_test.c:369-402
    toy_off = np.array([0, 3, 7], dtype=np.int32)
    toy_ptr, toy_ind = R.sparse_init(toy_idx, toy_off, 5)
    np.savez_compressed(os.path.join(HERE, "small_sparse.npz"), X=w.X, Y=w.Y, idx=s.indices, off=s.offsets,
                        dists=s.dists, radius=np.float64(s.radius), indptr=indptr, indices=indices,
                        weights=weights, data=data, data_unweighted_scaled=data_unw, data_ridge=data_ridge,
                        ridge_alpha=np.float64(1.0), toy_idx=toy_idx, toy_off=toy_off, toy_indptr=toy_ptr,
                        toy_indices=toy_ind)


def _ref_procrustes(X, Y, refl, scal):
    h = R.lib()
    Xc = np.ascontiguousarray(X)
    Yc = np.ascontiguousarray(Y)
    T = np.zeros((X.shape[1], X.shape[1]))
    tx = R.TMat(R._dp(Xc), X.shape[0], X.shape[1])
    ty = R.TMat(R._dp(Yc), Y.shape[0], Y.shape[1])
    tt = R.TMat(R._dp(T), T.shape[0], T.shape[1])
    assert h.ha_procrustes(ctypes.byref(tx), ctypes.byref(ty), ctypes.byref(tt), refl, scal) == 0
    return T


def _ref_ridge(X, Y, alpha):
    h = R.lib()
    Xc = np.ascontiguousarray(X)
    Yc = np.ascontiguousarray(Y)
    B = np.zeros((X.shape[1], Y.shape[1]))
    tx = R.TMat(R._dp(Xc), X.shape[0], X.shape[1])
    ty = R.TMat(R._dp(Yc), Y.shape[0], Y.shape[1])
    tb = R.TMat(R._dp(B), B.shape[0], B.shape[1])
    assert h.ha_ridge(ctypes.byref(tx), ctypes.byref(ty), float(alpha), ctypes.byref(tb)) == 0
    return B


def make_kat():
    out = {}
    X = O.SplitMix64(77).fill(50, 20)  # csrc/ha_test.c:234-256
    out["identity_X"] = X
    out["identity_T"] = _ref_procrustes(X, X, True, False)
    X = O.SplitMix64(55).fill(50, 10)  # csrc/ha_test.c:258-299
    Rm = np.eye(10)
    a = 0.7
    Rm[0, 0], Rm[0, 1], Rm[1, 0], Rm[1, 1] = np.cos(a), -np.sin(a), np.sin(a), np.cos(a)
    Y = X @ Rm
    out["rotation_X"], out["rotation_Y"] = X, Y
    out["rotation_T"] = _ref_procrustes(X, Y, True, False)
    g = O.SplitMix64(33)  # csrc/ha_test.c:301-334
    X = g.fill(50, 10)
    Y = g.fill(50, 10)
    out["noref_X"], out["noref_Y"] = X, Y
    out["noref_T"] = _ref_procrustes(X, Y, False, False)
    out["noref_scal_T"] = _ref_procrustes(X, Y, False, True)
    g = O.SplitMix64(101)  # csrc/ha_test.c:336-366
    X = g.fill(50, 10)
    B = g.fill(10, 5)
    Y = X @ B
    out["ridge_X"], out["ridge_Y"], out["ridge_B"] = X, Y, B
    out["ridge_betas"] = _ref_ridge(X, Y, 1e-6)
    np.savez_compressed(os.path.join(HERE, "kat.npz"), **out)


def make_grid():
    """CV splits (ha_ensemble_indices), ridge grid (ha_ridge_grid) and ensemble ridge
    (ha_ensemble_ridge) of the compiled reference on small seeded inputs."""
    out = {}
    tr, te = R.ensemble_indices(500, 1, 5, 10, 10, 5)
    out["cv_train"] = np.stack(tr)
    out["cv_test"] = np.concatenate(te)
    out["cv_test_sizes"] = np.array([t.size for t in te], dtype=np.int32)
    rng = np.random.default_rng(12)
    mask = rng.random(150) > 0.2
    tr, te = R.ensemble_indices(150, 2, 3, 7, 4, 9, mask)
    out["cvm_mask"] = mask
    out["cvm_train"] = np.stack(tr)
    out["cvm_test"] = np.concatenate(te)
    out["cvm_test_sizes"] = np.array([t.size for t in te], dtype=np.int32)
    X = rng.standard_normal((60, 10))
    y = X @ rng.standard_normal(10) + 0.5 * rng.standard_normal(60)
    alphas = np.logspace(-3, 3, 7)
    out["grid_X"], out["grid_y"], out["grid_alphas"] = X, y, alphas
    out["grid_npcs"] = np.array([2, 4, 20], dtype=np.int32)
    out["grid_npcs_odd"] = np.array([5, 3, 7, 0, 20], dtype=np.int32)
    boot = rng.integers(0, 60, 60).astype(np.int32)
    out["grid_boot"] = boot
    out["grid_betas"] = R.ridge_grid(X, y, alphas, out["grid_npcs"], boot)
    out["grid_betas_odd"] = R.ridge_grid(X, y, alphas, out["grid_npcs_odd"])
    tr, te = R.ensemble_indices(60, 1, 4, 5, 2, 3)
    out["ens_train"] = np.stack(tr)
    out["ens_test"] = np.concatenate(te)
    out["ens_test_sizes"] = np.array([t.size for t in te], dtype=np.int32)
    w, pred, r2, alpha, npc = R.ensemble_ridge(X, y, alphas, out["grid_npcs"], tr, te)
    out["ens_w"], out["ens_pred"] = w, pred
    out["ens_r2"], out["ens_alpha"], out["ens_npc"] = np.float64(r2), np.float64(alpha), np.int32(npc)
    np.savez_compressed(os.path.join(HERE, "grid.npz"), **out)


def make_python_ref():
    sys.path.insert(0, os.path.join(REF_DIR, "src"))
    from hyperalignment.procrustes import procrustes as py_procrustes  # noqa: E402
    from hyperalignment.sparse import initialize_sparse_matrix  # noqa: E402
    w = small_inputs(0)
    s = w.sls
    sls, _ = s.as_lists()
    Ts = [py_procrustes(w.X[:, sl], w.Y[:, sl], reflection=True, scaling=False) for sl in sls[:20]]
    mat = initialize_sparse_matrix(sls, nv=w.nv)
    np.savez_compressed(os.path.join(HERE, "python_ref.npz"), T_first20=np.concatenate([t.ravel() for t in Ts]),
                        indptr=mat.indptr.astype(np.int32), indices=mat.indices.astype(np.int32))


def make_pca_template():
    sys.path.insert(0, os.path.join(REF_DIR, "src"))
    from hyperalignment.searchlight import searchlight_template  # noqa: E402
    rng = np.random.default_rng(1)
    pts = W.fibonacci_sphere(162)
    sls = W.searchlights_knn(pts, rng.integers(8, 25, size=162))
    L = rng.standard_normal((60, 162))
    dms = np.stack([L + 0.01 * rng.standard_normal((60, 162)) for _ in range(4)])
    sl_list, d_list = sls.as_lists()
    tpl = searchlight_template(dms, sl_list, d_list, sls.radius, tpl_kind="pca")
    np.savez_compressed(os.path.join(HERE, "pca_template.npz"), dms=dms, idx=sls.indices, off=sls.offsets,
                        dists=sls.dists, radius=np.float64(sls.radius), template=tpl)


MAKERS = {"small_dense": make_small_dense, "small_sparse": make_small_sparse, "kat": make_kat, "grid": make_grid,
          "python_ref": make_python_ref, "pca_template": make_pca_template}

if __name__ == "__main__":
    names = sys.argv[1:] or list(MAKERS)
    if any(n in ("small_dense", "small_sparse", "kat", "grid") for n in names) and not R.available():
        raise SystemExit("build the reference first: make -C oracle")
    for n in names:
        MAKERS[n]()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
