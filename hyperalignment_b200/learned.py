"""The learned (alpha, PC count) proposal on top of the searchlight ridge grid search.

No reference counterpart: the reference only has the full grid search (csrc/ha_ridge.c:97-345).
The perceptron is trained on the GPU by the library's own kernels (ha_b200_mlp_*) on the
winners of the grid search for training subjects, and proposes the grid point of every
searchlight of a new subject from the searchlight's singular-value spectrum; the full grid search
stays as the fallback where the proposal's probability is below a threshold.

All device buffers are torch tensors (PyTorch is only the allocator here); every computation runs
in libha_b200.so.
"""

from __future__ import annotations

import ctypes
import dataclasses
import time

import numpy as np

from . import _lib as L
from . import workloads as W
from .plan import Plan

N_FEAT = 65


def _t(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def _dev_matrix(X):
    import torch
    return torch.from_numpy(np.asfortranarray(X).ravel(order="F")).cuda()


@dataclasses.dataclass
class Subject:
    """One subject pair of the grid workload, restricted to a searchlight subset, on the GPU."""
    w: W.Workload
    sls: W.Searchlights
    plan: Plan
    dX: object
    dY: object
    fit_rows: np.ndarray
    eval_rows: np.ndarray
    train_li: list
    test_li: list

    def close(self):
        self.plan.close()


def make_subject(seed, nv, nt=500, n_fit=400, step=1, size_lo=50, size_hi=500, noise=0.2, noise_span=30.0,
                 folds=5, blocksize=10, buffersize=10):
    """Subject pair of the grid workload with spatially varying noise (so the best grid point
    varies over the sphere), the first n_fit time points for fitting (CV splits of
    ha_ensemble_indices over them) and the rest for evaluation."""
    from . import hyperalignment_c as H
    w = W.ridge_grid_pair(seed, nv=nv, nt=nt, size_lo=size_lo, size_hi=size_hi, noise=noise, noise_span=noise_span)
    sls = w.sls.subset(np.arange(0, w.sls.count, step)) if step > 1 else w.sls
    plan = Plan(w.nt, w.nv, sls.indices, sls.offsets, sls.dists, sls.radius)
    tr, te = H.ensemble_indices(n_fit, 1, folds, blocksize, buffersize, seed)
    return Subject(w, sls, plan, _dev_matrix(w.X), _dev_matrix(w.Y), np.arange(n_fit, dtype=np.int32),
                   np.arange(n_fit, nt, dtype=np.int32), tr, te)


def grid_labels(sub, alphas=W.GRID_ALPHAS, npcs=W.GRID_NPCS):
    """Full grid search: (CSC values, winners, device milliseconds)."""
    import torch
    vals = torch.zeros(sub.plan.nnz, dtype=torch.float64, device="cuda")
    best = torch.zeros(sub.sls.count, dtype=torch.int32, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    sub.plan.ridge_grid_device(sub.dX.data_ptr(), sub.dY.data_ptr(), vals.data_ptr(), best.data_ptr(), alphas, npcs,
                               sub.train_li, sub.test_li)
    e1.record()
    torch.cuda.synchronize()
    return vals, best, e0.elapsed_time(e1)


def features(sub):
    import torch
    f = torch.zeros((sub.sls.count, N_FEAT), dtype=torch.float32, device="cuda")
    sub.plan.ridge_features_device(sub.dX.data_ptr(), sub.fit_rows, f.data_ptr())
    torch.cuda.synchronize()
    return f


def train(feats, labels, n_classes, epochs=40, batch=128, lr=2e-3, seed=0):
    """Train the perceptron on the GPU; returns (parameters, final mean loss)."""
    import torch
    lib = L.lib()
    P = lib.ha_b200_mlp_param_count(n_classes)
    prm = torch.zeros(P, dtype=torch.float32, device="cuda")
    L.check(lib.ha_b200_mlp_init(ctypes.c_void_p(prm.data_ptr()), n_classes, seed), "ha_b200_mlp_init")
    loss = ctypes.c_float()
    L.check(lib.ha_b200_mlp_train(ctypes.c_void_p(prm.data_ptr()), n_classes, ctypes.c_void_p(feats.data_ptr()),
                                  ctypes.c_void_p(labels.data_ptr()), int(feats.shape[0]), epochs, batch, lr, seed,
                                  ctypes.byref(loss)), "ha_b200_mlp_train")
    return prm, loss.value


def learned(sub, prm, min_prob=0.6, alphas=W.GRID_ALPHAS, npcs=W.GRID_NPCS):
    """Learned form: (CSC values, chosen grid points, probabilities, device milliseconds)."""
    import torch
    vals = torch.zeros(sub.plan.nnz, dtype=torch.float64, device="cuda")
    choice = torch.zeros(sub.sls.count, dtype=torch.int32, device="cuda")
    prob = torch.zeros(sub.sls.count, dtype=torch.float32, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    sub.plan.ridge_learned_device(sub.dX.data_ptr(), sub.dY.data_ptr(), sub.fit_rows, alphas, npcs, prm.data_ptr(),
                                  min_prob, sub.train_li, sub.test_li, vals.data_ptr(), choice.data_ptr(),
                                  prob.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    return vals, choice, prob, e0.elapsed_time(e1)


def heldout_correlation(sub, vals):
    """Mean over vertices of the correlation between X_eval @ W and Y_eval (W: the scattered
    betas in CSC order), over vertices whose prediction varies."""
    import scipy.sparse as sp
    indptr, indices = sub.plan.pattern()
    Wm = sp.csc_matrix((vals.cpu().numpy(), indices, indptr), shape=(sub.w.nv, sub.w.nv))
    Xe = sub.w.X[sub.eval_rows]
    Ye = sub.w.Y[sub.eval_rows]
    pred = np.asarray(Xe @ Wm)
    pc = pred - pred.mean(0)
    yc = Ye - Ye.mean(0)
    den = np.sqrt((pc * pc).sum(0) * (yc * yc).sum(0))
    ok = den > 0
    return float(np.mean((pc * yc).sum(0)[ok] / den[ok]))


def study(train_seeds=(1, 2, 3, 4), test_seed=5, nv=10242, step=4, size_lo=50, size_hi=500, epochs=40,
          min_prob=0.6, log=print, train_step=None):
    """The learned-proposal study: labels from the full grid on the training subjects (every
    train_step-th searchlight, default step), training on the GPU, then the held-out subject (every
    step-th searchlight) through both the full grid and the learned form."""
    train_step = step if train_step is None else train_step
    import torch
    C = len(W.GRID_ALPHAS) * len(W.GRID_NPCS)
    feats, labels = [], []
    t0 = time.time()
    for sd in train_seeds:
        sub = make_subject(sd, nv, step=train_step, size_lo=size_lo, size_hi=size_hi)
        _, best, ms = grid_labels(sub)
        feats.append(features(sub))
        labels.append(best)
        log(f"seed {sd}: {sub.sls.count} searchlights, grid {ms:.0f} ms, "
            f"{len(np.unique(best.cpu().numpy()))} distinct winners")
        sub.close()
    F = torch.cat(feats)
    Y = torch.cat(labels)
    prm, loss = train(F, Y, C, epochs=epochs)
    log(f"trained on {F.shape[0]} searchlights, final loss {loss:.4f} ({time.time() - t0:.0f} s so far)")
    sub = make_subject(test_seed, nv, step=step, size_lo=size_lo, size_hi=size_hi)
    gvals, gbest, gms = grid_labels(sub)
    gvals2, gbest2, gms2 = grid_labels(sub)  # second run: warm
    # the plain FP32 form of the same full grid search (warm run timed)
    sub.plan.set_grid_precision(32)
    grid_labels(sub)
    fvals32, fbest32, fms32 = grid_labels(sub)
    sub.plan.set_grid_precision(64)
    lvals, choice, prob, lms = learned(sub, prm, min_prob)
    lvals, choice, prob, lms = learned(sub, prm, min_prob)
    # the mixed-precision learned form: float32 eigen solve, features, proposal fit and fallback
    # grid, bf16 inference (warm run timed)
    sub.plan.set_grid_precision(32)
    learned(sub, prm, min_prob)
    mvals, mchoice, mprob, mms = learned(sub, prm, min_prob)
    sub.plan.set_grid_precision(64)
    mp = mprob.cpu().numpy()
    p = prob.cpu().numpy()
    ch = choice.cpu().numpy()
    gb = gbest2.cpu().numpy()
    conf = p >= min_prob
    res = {
        "searchlights": int(sub.sls.count),
        "grid": {"ms": gms2, "searchlights_per_s": sub.sls.count / gms2 * 1e3,
                 "heldout_corr": heldout_correlation(sub, gvals2)},
        "grid_fp32": {"ms": fms32, "searchlights_per_s": sub.sls.count / fms32 * 1e3,
                      "heldout_corr": heldout_correlation(sub, fvals32),
                      "winners_equal_fp64": float((fbest32.cpu().numpy() == gb).mean())},
        "learned": {"ms": lms, "searchlights_per_s": sub.sls.count / lms * 1e3,
                    "heldout_corr": heldout_correlation(sub, lvals), "fallback": int((~conf).sum()),
                    "proposal_matches_grid": float((ch[conf] == gb[conf]).mean()) if conf.any() else None},
        "learned_fp32": {"ms": mms, "searchlights_per_s": sub.sls.count / mms * 1e3,
                         "heldout_corr": heldout_correlation(sub, mvals), "fallback": int((mp < min_prob).sum()),
                         "choices_equal_fp64_learned": float((mchoice.cpu().numpy() == ch).mean())},
        "train": {"examples": int(F.shape[0]), "final_loss": loss, "epochs": epochs},
    }
    # the method without the network: one fixed grid point (the training winners' mode)
    mode = int(np.bincount(Y.cpu().numpy(), minlength=C).argmax())
    zero = torch.zeros_like(prm)
    L.check(L.lib().ha_b200_mlp_init(ctypes.c_void_p(zero.data_ptr()), C, 0), "ha_b200_mlp_init")
    zero.zero_()
    lay = _layout(C)
    zero[lay["b3"]:lay["b3"] + C] = -30.0
    zero[lay["b3"] + mode] = 30.0
    fvals, _, _, fms = learned(sub, zero, 0.5)
    res["fixed_point"] = {"grid_point": mode, "ms": fms, "heldout_corr": heldout_correlation(sub, fvals)}
    sub.close()
    return res


def _layout(C):
    o, out = 0, {}
    for k, n in (("W1", 65 * 128), ("b1", 128), ("W2", 128 * 128), ("b2", 128), ("W3", 128 * C), ("b3", C)):
        out[k] = o
        o += n
    return out
