"""The learned form of the ridge grid search through the C ABI (plan device entries).

Checks, against the CPU oracle on small cases:
  * features (singular values of the fit rows / the largest, log n): relative 1e-5 (float32)
  * a confident proposal gives ha_ridge_grid's beta at the proposed grid point, fitted on the fit
    rows (csrc/ha_ridge.c:97-227): relative 1e-8
  * below the probability threshold the full CV grid search runs: identical to the grid entry
  * a mix of both goes through the fallback mask correctly
  * the same with the plan's grid precision at 32 (float32 eigen solve, fit and fallback grid):
    features 1e-4, the proposal's fit 1e-4, the fallback identical to the float32 grid entry
"""

import ctypes

import numpy as np
import pytest

from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import learned as LR
from hyperalignment_b200 import workloads as W
from oracle import ha_oracle as O

pytestmark = pytest.mark.gpu

ALPHAS = np.logspace(-2, 3, 4)
NPCS = np.array([5, 12, 1 << 30], dtype=np.int32)
C = ALPHAS.size * NPCS.size


def relf(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def sub(gpu):
    s = LR.make_subject(3, nv=642, nt=120, n_fit=96, step=3, size_lo=8, size_hi=60, noise_span=30.0, blocksize=6,
                        buffersize=3, folds=4)
    yield s
    s.close()


def _forced(g, logit=30.0):
    import torch
    lay = LR._layout(C)
    prm = torch.zeros(L.lib().ha_b200_mlp_param_count(C), dtype=torch.float32, device="cuda")
    prm[lay["b3"]:lay["b3"] + C] = -logit
    prm[lay["b3"] + g] = logit
    return prm


def _run_learned(sub, prm, min_prob):
    import torch
    vals = torch.zeros(sub.plan.nnz, dtype=torch.float64, device="cuda")
    choice = torch.zeros(sub.sls.count, dtype=torch.int32, device="cuda")
    prob = torch.zeros(sub.sls.count, dtype=torch.float32, device="cuda")
    sub.plan.ridge_learned_device(sub.dX.data_ptr(), sub.dY.data_ptr(), sub.fit_rows, ALPHAS, NPCS, prm.data_ptr(),
                                  min_prob, sub.train_li, sub.test_li, vals.data_ptr(), choice.data_ptr(),
                                  prob.data_ptr())
    torch.cuda.synchronize()
    return vals.cpu().numpy(), choice.cpu().numpy(), prob.cpu().numpy()


def _oracle_at(sub, choice, which):
    s = sub.sls
    indptr, indices = sub.plan.pattern()
    data = np.zeros(indices.size)
    wts = O.searchlight_weights(s.indices, s.offsets, s.dists, s.radius, sub.w.nv)
    for q in np.flatnonzero(which):
        sl = s.indices[s.offsets[q]:s.offsets[q + 1]]
        a, p = divmod(int(choice[q]), NPCS.size)
        B = O.ridge_grid(sub.w.X[:, sl], sub.w.Y[:, sl], ALPHAS, NPCS, sub.fit_rows)[:, a, p, :]
        O.sparse_scatter_add(indptr, indices, data, sl, sl, B, wts[s.offsets[q]:s.offsets[q + 1]])
    return data


def test_features_match_oracle(sub):
    f = LR.features(sub).cpu().numpy().astype(np.float64)
    ref = O.ridge_features(sub.w.X, sub.sls.indices, sub.sls.offsets, sub.fit_rows)
    assert relf(f, ref) <= 1e-5


def test_confident_proposal_is_the_grid_point_fit(sub):
    g = 7
    vals, choice, prob = _run_learned(sub, _forced(g), 0.5)
    assert (choice == g).all() and (prob > 0.99).all()
    ref = _oracle_at(sub, choice, np.ones(sub.sls.count, dtype=bool))
    assert relf(vals, ref) <= 1e-8


def test_fallback_is_the_full_grid(sub):
    gvals, gbest, _ = LR.grid_labels(sub, ALPHAS, NPCS)
    vals, choice, prob = _run_learned(sub, _forced(2), 2.0)  # no proposal reaches probability 2
    assert np.array_equal(vals, gvals.cpu().numpy())
    assert np.array_equal(choice, gbest.cpu().numpy())


def test_mixed_proposals_and_fallbacks(sub):
    import torch
    # a random network: probabilities spread around the threshold
    prm = torch.zeros(L.lib().ha_b200_mlp_param_count(C), dtype=torch.float32, device="cuda")
    assert L.lib().ha_b200_mlp_init(ctypes.c_void_p(prm.data_ptr()), C, 5) == 0
    prm *= 8.0
    _, _, p0 = _run_learned(sub, prm, 2.0)
    thr = float(np.median(p0))
    vals, choice, prob = _run_learned(sub, prm, thr)
    conf = prob >= thr
    assert 0 < conf.sum() < conf.size
    gvals, gbest, _ = LR.grid_labels(sub, ALPHAS, NPCS)
    gb = gbest.cpu().numpy()
    assert np.array_equal(choice[~conf], gb[~conf])
    # oracle: the proposal's fit where confident plus the grid winner's betas elsewhere
    s = sub.sls
    indptr, indices = sub.plan.pattern()
    ref = _oracle_at(sub, choice, conf)
    fb = np.flatnonzero(~conf)
    sub_sls = s.subset(fb)
    wts = O.searchlight_weights(s.indices, s.offsets, s.dists, s.radius, sub.w.nv)
    wsub = np.concatenate([wts[s.offsets[q]:s.offsets[q + 1]] for q in fb])
    d2, rbest, _ = O.searchlight_ridge_grid_csc(sub.w.X, sub.w.Y, sub_sls.indices, sub_sls.offsets, indptr, indices,
                                                np.zeros(indices.size), ALPHAS, NPCS, sub.train_li, sub.test_li, wsub)
    if np.array_equal(rbest, gb[~conf]):
        assert relf(vals, ref + d2) <= 1e-8


# ---- the mixed-precision learned form: float32 eigen solve, proposal fit and fallback grid ----

@pytest.fixture
def fp32(sub):
    sub.plan.set_grid_precision(32)
    yield sub
    sub.plan.set_grid_precision(64)


def test_fp32_features_match_oracle(fp32):
    # the network's input: singular values over the largest from the float32 eigen solve
    f = LR.features(fp32).cpu().numpy().astype(np.float64)
    ref = O.ridge_features(fp32.w.X, fp32.sls.indices, fp32.sls.offsets, fp32.fit_rows)
    assert relf(f, ref) <= 1e-4


def test_fp32_confident_proposal_is_the_grid_point_fit(fp32):
    g = 7
    vals, choice, prob = _run_learned(fp32, _forced(g), 0.5)
    assert (choice == g).all() and (prob > 0.99).all()
    ref = _oracle_at(fp32, choice, np.ones(fp32.sls.count, dtype=bool))
    assert relf(vals, ref) <= 1e-4


def test_fp32_fallback_is_the_fp32_full_grid(fp32):
    gvals, gbest, _ = LR.grid_labels(fp32, ALPHAS, NPCS)
    vals, choice, prob = _run_learned(fp32, _forced(2), 2.0)
    assert np.array_equal(vals, gvals.cpu().numpy())
    assert np.array_equal(choice, gbest.cpu().numpy())
