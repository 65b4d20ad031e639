"""Pins the CPU oracle (oracle/ha_oracle.py) to the reference.

Known-answer tests restate csrc/ha_test.c (same splitmix64 / Box-Muller inputs);
golden comparisons use outputs of the compiled reference and of the Python
reference package stored in tests/golden/ (made by tests/golden/make_golden.py).
"""

import numpy as np
import pytest

from conftest import golden
from oracle import ha_oracle as O


def test_kat_procrustes_identity():
    # csrc/ha_test.c:234-256: |T| ~ I within 1e-8
    g = golden("kat.npz")
    X = O.SplitMix64(77).fill(50, 20)
    np.testing.assert_array_equal(X, g["identity_X"])
    T = O.procrustes(X, X, True, False)
    np.testing.assert_allclose(np.abs(T), np.eye(20), atol=1e-8)
    np.testing.assert_allclose(T, g["identity_T"], atol=1e-10)


def test_kat_procrustes_known_rotation():
    # csrc/ha_test.c:258-299: ||X T - Y||_inf < 1e-8
    g = golden("kat.npz")
    X = O.SplitMix64(55).fill(50, 10)
    np.testing.assert_array_equal(X, g["rotation_X"])
    T = O.procrustes(X, g["rotation_Y"], True, False)
    assert np.abs(X @ T - g["rotation_Y"]).max() < 1e-8
    np.testing.assert_allclose(T, g["rotation_T"], atol=1e-10)


def test_kat_procrustes_no_reflection():
    # csrc/ha_test.c:301-334: det(T) > 0
    g = golden("kat.npz")
    T = O.procrustes(g["noref_X"], g["noref_Y"], False, False)
    assert np.linalg.det(T) > 0
    np.testing.assert_allclose(T, g["noref_T"], atol=1e-10)
    Ts = O.procrustes(g["noref_X"], g["noref_Y"], False, True)
    np.testing.assert_allclose(Ts, g["noref_scal_T"], atol=1e-10)


def test_kat_ridge_small_alpha():
    # csrc/ha_test.c:336-366: betas recovered within 1e-6
    g = golden("kat.npz")
    B = O.ridge(g["ridge_X"], g["ridge_Y"], 1e-6)
    assert np.abs(B - g["ridge_B"]).max() < 1e-6
    np.testing.assert_allclose(B, g["ridge_betas"], atol=1e-10)


def test_kat_sparse_init_toy():
    # csrc/ha_test.c:369-402: two overlapping searchlights on 5 vertices -> nnz 21
    g = golden("small_sparse.npz")
    indptr, indices = O.sparse_init(g["toy_idx"], g["toy_off"], 5)
    assert indices.size == 21
    np.testing.assert_array_equal(indptr, g["toy_indptr"])
    np.testing.assert_array_equal(indices, g["toy_indices"])


def test_kat_sparse_scatter_identity():
    # csrc/ha_test.c:404-435
    sl = np.array([0, 1, 2], dtype=np.int32)
    indptr, indices = O.sparse_init(sl, np.array([0, 3], dtype=np.int32), 3)
    data = np.zeros(indices.size)
    O.sparse_scatter_add(indptr, indices, data, sl, sl, np.eye(3))
    cols = np.repeat(np.arange(3), np.diff(indptr))
    np.testing.assert_array_equal(data, (indices == cols).astype(float))


def test_kat_weights_sum_to_one():
    # csrc/ha_test.c:439-470 (uniform weights)
    idx = np.array([0, 1, 2, 1, 2, 3, 4, 3, 4, 5], dtype=np.int32)
    off = np.array([0, 3, 7, 10], dtype=np.int32)
    w = O.searchlight_weights(idx, off, None, 0.0, 6)
    sums = np.zeros(6)
    np.add.at(sums, idx, w)
    np.testing.assert_allclose(sums, 1.0, atol=1e-12)


def test_kat_zscore():
    # csrc/ha_test.c:474-500
    X = O.zscore_columns(O.SplitMix64(200).fill(100, 10))
    np.testing.assert_allclose(X.mean(axis=0), 0.0, atol=1e-12)
    np.testing.assert_allclose((X * X).mean(axis=0) - X.mean(axis=0) ** 2, 1.0, atol=1e-10)


def test_weights_bit_exact_vs_reference():
    g = golden("small_sparse.npz")
    w = O.searchlight_weights(g["idx"], g["off"], g["dists"], float(g["radius"]), g["X"].shape[1])
    np.testing.assert_array_equal(w, g["weights"])


def test_sparse_pattern_bit_exact_vs_reference():
    g = golden("small_sparse.npz")
    indptr, indices = O.sparse_init(g["idx"], g["off"], g["X"].shape[1])
    np.testing.assert_array_equal(indptr, g["indptr"])
    np.testing.assert_array_equal(indices, g["indices"])


def test_sparse_pattern_matches_python_reference():
    g = golden("python_ref.npz")
    d = golden("small_dense.npz")
    indptr, indices = O.sparse_init(d["idx"], d["off"], d["X"].shape[1])
    np.testing.assert_array_equal(indptr, g["indptr"])
    np.testing.assert_array_equal(indices, g["indices"])


def test_procrustes_matches_python_reference():
    g = golden("python_ref.npz")
    d = golden("small_dense.npz")
    Ts = O.local_transforms(d["X"], d["Y"], d["idx"], d["off"][:21])
    np.testing.assert_allclose(np.concatenate([t.ravel() for t in Ts]), g["T_first20"], atol=1e-10)


@pytest.mark.parametrize("key,refl,scal,weighted", [
    ("T_cpu64", True, False, True),
    ("T_cpu64_noref_scal", False, True, True),
    ("T_cpu64_uniform", True, False, False),
])
def test_dense_matches_reference(key, refl, scal, weighted):
    g = golden("small_dense.npz")
    dists = g["dists"] if weighted else None
    T = O.searchlight_procrustes_dense(g["X"], g["Y"], g["idx"], g["off"], dists, float(g["radius"]), refl, scal)
    np.testing.assert_allclose(T, g[key], atol=1e-10, rtol=0)


def test_dense_cpu32_close_to_cpu64():
    # the reference's own FP32 arm sits within ~1e-6 of FP64 on this case
    g = golden("small_dense.npz")
    a, b = g["T_cpu64"], g["T_cpu32"]
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-5


def test_sparse_procrustes_and_ridge_match_reference():
    g = golden("small_sparse.npz")
    X, Y, idx, off = g["X"], g["Y"], g["idx"], g["off"]
    d = O.searchlight_procrustes_csc(X, Y, idx, off, g["indptr"], g["indices"], np.zeros(g["indices"].size),
                                     g["weights"], True, False)
    np.testing.assert_allclose(d, g["data"], atol=1e-10, rtol=0)
    d = O.searchlight_procrustes_csc(X, Y, idx, off, g["indptr"], g["indices"], np.zeros(g["indices"].size),
                                     None, True, True)
    np.testing.assert_allclose(d, g["data_unweighted_scaled"], atol=1e-10, rtol=0)
    d = O.searchlight_ridge_csc(X, Y, idx, off, g["indptr"], g["indices"], np.zeros(g["indices"].size),
                                float(g["ridge_alpha"]), g["weights"])
    np.testing.assert_allclose(d, g["data_ridge"], atol=1e-10, rtol=0)


def test_oracle_vs_live_reference():
    """When the compiled reference is present (oracle/_ref), compare on a fresh seed."""
    from oracle import ref_lib as R
    if not R.available():
        pytest.skip("compiled reference not built (make -C oracle)")
    from hyperalignment_b200 import workloads as W
    w = W.small_case(seed=7, reflection=False, scaling=True)
    s = w.sls
    a = O.searchlight_procrustes_dense(w.X, w.Y, s.indices, s.offsets, s.dists, s.radius, False, True)
    b = R.procrustes_dense(w.X, w.Y, s.indices, s.offsets, s.dists, s.radius, False, True, 0, threads=1)
    np.testing.assert_allclose(a, b, atol=1e-10, rtol=0)


def test_template_identical_subjects_oracle():
    """Searchlight form of csrc/ha_test.c:503-537: identical subjects give the input back."""
    from hyperalignment_b200 import workloads as W
    _, sls, subj = W.hemisphere_subjects(seed=4, nv=162, nt=60, n_subj=3, size_lo=8, size_hi=20)
    base = subj[0]
    tpl = O.searchlight_template([base, base.copy(), base.copy()], sls.indices, sls.offsets, sls.dists, sls.radius,
                                 True, False, False, 1)
    assert np.abs(tpl - base).max() < 1e-8


def _split(g, pre):
    sizes = g[pre + "_test_sizes"]
    test = np.split(g[pre + "_test"], np.cumsum(sizes)[:-1])
    return list(g[pre + "_train"]), test


@pytest.mark.parametrize("pre,args,mask", [
    ("cv", (500, 1, 5, 10, 10, 5), False),   # the temporally blocked 5-fold layout of the grid search
    ("cvm", (150, 2, 3, 7, 4, 9), True),     # two permutations, masked time points, remapped indices
])
def test_ensemble_indices_bit_exact(pre, args, mask):
    # csrc/ha_ensemble.c:58-249 draw for draw (xoshiro256** / splitmix64, modulo sampling)
    g = golden("grid.npz")
    tr, te = O.ensemble_indices(*args, mask=g["cvm_mask"] if mask else None)
    rtr, rte = _split(g, pre)
    assert len(tr) == len(rtr)
    for a, b in zip(tr + te, rtr + rte):
        np.testing.assert_array_equal(a, b)


def test_ensemble_test_sets_overlap():
    # buffer rows next to a test block can be tested by two folds: the ensemble averages them
    g = golden("grid.npz")
    _, te = _split(g, "cv")
    count = np.zeros(500, dtype=int)
    for t in te:
        count[t] += 1
    assert count.max() >= 2


def test_ridge_grid_matches_reference():
    # csrc/ha_ridge.c:97-227: PC chunks clipped at K, cumulative over p; bootstrap training rows
    g = golden("grid.npz")
    B = O.ridge_grid(g["grid_X"], g["grid_y"], g["grid_alphas"], g["grid_npcs"], g["grid_boot"])
    np.testing.assert_allclose(B, g["grid_betas"], atol=1e-12, rtol=0)
    # non-monotone PC counts: empty chunks and double-counted components as the reference sums them
    B = O.ridge_grid(g["grid_X"], g["grid_y"], g["grid_alphas"], g["grid_npcs_odd"])
    np.testing.assert_allclose(B, g["grid_betas_odd"], atol=1e-12, rtol=0)


def test_ensemble_ridge_matches_reference():
    # csrc/ha_ridge.c:229-345: averaged test predictions, first argmin, r2
    g = golden("grid.npz")
    tr, te = _split(g, "ens")
    w, pred, r2, alpha, npc, best, cost = O.ensemble_ridge(g["grid_X"], g["grid_y"], g["grid_alphas"],
                                                           g["grid_npcs"], tr, te)
    np.testing.assert_allclose(w, g["ens_w"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(pred, g["ens_pred"], atol=1e-12, rtol=0)
    assert abs(r2 - float(g["ens_r2"])) < 1e-12
    assert alpha == float(g["ens_alpha"]) and npc == int(g["ens_npc"])
    assert cost.shape == (g["grid_alphas"].size, g["grid_npcs"].size)


def test_ensemble_ridge_multi_target_sums_costs():
    # the searchlight composition: one winner per searchlight, cost summed over its targets
    g = golden("grid.npz")
    tr, te = _split(g, "ens")
    X = g["grid_X"]
    Y = np.stack([g["grid_y"], X[:, 0] - X[:, 3], X[:, 5]], axis=1)
    *_, cost = O.ensemble_ridge(X, Y, g["grid_alphas"], g["grid_npcs"], tr, te)
    per = sum(O.ensemble_ridge(X, Y[:, k], g["grid_alphas"], g["grid_npcs"], tr, te)[6] for k in range(3))
    np.testing.assert_allclose(cost, per, rtol=1e-12)


def test_grid_oracle_vs_live_reference():
    from oracle import ref_lib as R
    if not R.available():
        pytest.skip("compiled reference not built (make -C oracle)")
    rng = np.random.default_rng(3)
    X = rng.standard_normal((90, 14))
    y = X @ rng.standard_normal(14) + rng.standard_normal(90)
    al, npcs = np.logspace(-2, 2, 4), [3, 8, 100]
    tr, te = R.ensemble_indices(90, 1, 3, 6, 3, 21)
    a = O.ensemble_ridge(X, y, al, npcs, tr, te)
    b = R.ensemble_ridge(X, y, al, npcs, tr, te)
    np.testing.assert_allclose(a[0], b[0], atol=1e-12, rtol=0)
    assert (a[3], a[4]) == (b[3], b[4])


def test_mlp_oracle_gradient_vs_finite_differences():
    # the perceptron of the learned proposal has no reference counterpart: its float64 restatement
    # is checked against central differences before it checks the GPU kernels
    rng = np.random.default_rng(0)
    C = 7
    P = O.mlp_layout(C)["total"]
    params = rng.uniform(-0.3, 0.3, P)
    X = rng.standard_normal((9, O.MLP_IN))
    y = rng.integers(0, C, 9)
    loss, g = O.mlp_loss_grad(params, C, X, y)
    for k in rng.choice(P, 40, replace=False):
        e = np.zeros(P)
        e[k] = 1e-6
        fd = (O.mlp_loss_grad(params + e, C, X, y)[0] - O.mlp_loss_grad(params - e, C, X, y)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-7 + 1e-5 * abs(g[k]), (k, fd, g[k])
    assert np.isclose(loss, np.mean(np.log(np.exp(O.mlp_forward(params, C, X)).sum(1))
                                    - O.mlp_forward(params, C, X)[np.arange(9), y]))


# ---------------------------------------------------------------------------------------------
# the restatement against the compiled reference on fresh seeds (skipped when it is not built)
# ---------------------------------------------------------------------------------------------

def _ref():
    from oracle import ref_lib as R
    if not R.available():
        pytest.skip("compiled reference not built (make -C oracle)")
    return R


@pytest.mark.parametrize("refl,scal,weighted", [(True, False, True), (False, False, True), (True, True, False),
                                               (False, True, True)])
def test_dense_procrustes_vs_live_reference(refl, scal, weighted):
    R = _ref()
    from hyperalignment_b200 import workloads as W
    w = W.small_case(seed=41, nv=162, nt=50, lo=6, hi=30)
    s = w.sls
    d = s.dists if weighted else None
    a = O.searchlight_procrustes_dense(w.X, w.Y, s.indices, s.offsets, d, s.radius, refl, scal)
    b = R.procrustes_dense(w.X, w.Y, s.indices, s.offsets, d, s.radius, refl, scal, 0, threads=1)
    np.testing.assert_allclose(a, b, atol=1e-10, rtol=0)


@pytest.mark.parametrize("alpha", [1e-3, 1.0, 100.0])
def test_sparse_procrustes_and_ridge_vs_live_reference(alpha):
    R = _ref()
    from hyperalignment_b200 import workloads as W
    w = W.small_case(seed=43, nv=162, nt=40, lo=6, hi=24)
    s = w.sls
    indptr, indices = O.sparse_init(s.indices, s.offsets, w.nv)
    ri, rj = R.sparse_init(s.indices, s.offsets, w.nv)
    np.testing.assert_array_equal(indptr, ri)
    np.testing.assert_array_equal(indices, rj)
    wts = O.searchlight_weights(s.indices, s.offsets, s.dists, s.radius, w.nv)
    np.testing.assert_array_equal(wts, R.searchlight_weights(s.indices, s.offsets, s.dists, s.radius))
    a = O.searchlight_ridge_csc(w.X, w.Y, s.indices, s.offsets, indptr, indices, np.zeros(indices.size), alpha, wts)
    b = R.searchlight_ridge_csc(w.X, w.Y, s.indices, s.offsets, indptr, indices, alpha, wts, threads=1)
    np.testing.assert_allclose(a, b, atol=1e-10 * max(1.0, np.abs(b).max()), rtol=0)
    a = O.searchlight_procrustes_csc(w.X, w.Y, s.indices, s.offsets, indptr, indices, np.zeros(indices.size), wts,
                                     True, False)
    b = R.searchlight_procrustes_csc(w.X, w.Y, s.indices, s.offsets, indptr, indices, wts, True, False, threads=1)
    np.testing.assert_allclose(a, b, atol=1e-10, rtol=0)


@pytest.mark.parametrize("args", [(300, 3, 4, 8, 0, 11), (97, 2, 3, 5, 2, 0), (64, 1, 2, 16, 4, 123456789)])
def test_ensemble_indices_vs_live_reference(args):
    R = _ref()
    tr, te = O.ensemble_indices(*args)
    rtr, rte = R.ensemble_indices(*args)
    assert len(tr) == len(rtr)
    for a, b in zip(tr + te, rtr + rte):
        np.testing.assert_array_equal(a, b)


def test_aligned_correlation_restatement():
    """The evaluation of benchmark_neuroboros.py:204-211 against per-column Pearson correlation,
    with X @ W for a sparse W, and NaN for a constant column (scipy's z-score divides 0 by 0)."""
    import scipy.sparse as sp
    rng = np.random.default_rng(4)
    X = rng.standard_normal((50, 12))
    Y = rng.standard_normal((50, 12))
    W = sp.random(12, 12, density=0.4, random_state=5, format="csc") + sp.identity(12, format="csc")
    A = np.asarray(X @ W)
    r = O.aligned_correlation(X, Y, W)
    want = np.array([np.corrcoef(A[:, j], Y[:, j])[0, 1] for j in range(12)])
    np.testing.assert_allclose(r, want, rtol=0, atol=1e-12)
    np.testing.assert_allclose(O.aligned_correlation(X, Y), [np.corrcoef(X[:, j], Y[:, j])[0, 1] for j in range(12)],
                               rtol=0, atol=1e-12)
    Y[:, 3] = 2.5
    r = O.aligned_correlation(X, Y, W)
    assert np.isnan(r[3]) and np.isfinite(np.delete(r, 3)).all()


def test_pca_template_restatement_vs_python_reference():
    """searchlight_template(tpl_kind="pca") of the Python reference on subjects whose searchlights
    have a separated top singular subspace: the exact-SVD restatement agrees with the reference's
    randomized SVD there (the fixture is made by tests/golden/make_golden.py)."""
    g = golden("pca_template.npz")
    tpl = O.searchlight_pca_template(list(g["dms"]), g["idx"], g["off"], g["dists"], float(g["radius"]))
    assert np.linalg.norm(tpl - g["template"]) <= 1e-12 * np.linalg.norm(g["template"])


@pytest.mark.parametrize("refl,scal,zs,level2", [(True, False, True, 1), (False, True, False, 2), (True, True, True, 0)])
def test_template_loop_vs_live_reference(refl, scal, zs, level2):
    """The template loop restated around searchlight solves reduces, for one searchlight holding
    every vertex (weight 1), to the reference's whole-matrix ha_template_procrustes
    (csrc/ha_template.c:14-114): same running average, leave-one-out passes, z-scores and final
    sum."""
    from oracle import ref_lib as R
    if not R.available():
        pytest.skip("compiled reference not built (make -C oracle)")
    rng = np.random.default_rng(3)
    nt, nv, ns = 30, 12, 4
    L = rng.standard_normal((nt, nv))
    dms = []
    for _ in range(ns):
        Q, r = np.linalg.qr(rng.standard_normal((nv, nv)))
        dms.append(L @ (Q * np.sign(np.diag(r))) + 0.3 * rng.standard_normal((nt, nv)))
    ref = R.template_procrustes(dms, refl, scal, zs, level2)
    ours = O.searchlight_template(dms, np.arange(nv, dtype=np.int32), np.array([0, nv], dtype=np.int32), None, 0.0,
                                  refl, scal, zs, level2)
    assert np.linalg.norm(ours - ref) <= 1e-12 * np.linalg.norm(ref)
