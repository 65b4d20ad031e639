"""Plans whose scratch does not fit the budget run chunk by chunk (a full 40962-vertex grid
search needs several chunks).  A tiny budget forces many chunks here; the results must match the
single-chunk plan: per-chunk reductions add in a different order, so within 1e-12 relative, and
the grid winners identical."""

import os

import numpy as np
import pytest

from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import hyperalignment_c as H
from hyperalignment_b200 import workloads as W
from hyperalignment_b200.plan import Plan

pytestmark = pytest.mark.gpu


def _run(w, Y, tr, te, budget_gb):
    import torch
    old = os.environ.get("HA_B200_SCRATCH_GB")
    os.environ["HA_B200_SCRATCH_GB"] = budget_gb
    try:
        s = w.sls
        plan = Plan(w.nt, w.nv, s.indices, s.offsets, s.dists, s.radius)
        dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).cuda()
        dY = torch.from_numpy(np.asfortranarray(Y).ravel(order="F")).cuda()
        out = {}
        for name, solver in (("mixed", L.SOLVER_MIXED), ("fp32", L.SOLVER_FP32)):
            v = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
            plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), v.data_ptr(), True, True, solver, L.OUT_CSC)
            torch.cuda.synchronize()
            out[name] = v.cpu().numpy()
        v = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
        best = torch.zeros(s.count, dtype=torch.int32, device="cuda")
        plan.ridge_grid_device(dX.data_ptr(), dY.data_ptr(), v.data_ptr(), best.data_ptr(), [1e-2, 1.0, 100.0],
                               [5, 1 << 30], tr, te)
        torch.cuda.synchronize()
        out["grid"], out["best"] = v.cpu().numpy(), best.cpu().numpy()
        plan.close()
        return out
    finally:
        if old is None:
            del os.environ["HA_B200_SCRATCH_GB"]
        else:
            os.environ["HA_B200_SCRATCH_GB"] = old


def test_many_chunks_match_one(gpu):
    w = W.small_case(seed=17, nv=642, nt=120, lo=20, hi=70)
    Y = 0.5 * w.Y + np.random.default_rng(3).standard_normal(w.Y.shape)
    tr, te = H.ensemble_indices(120, 1, 4, 6, 3, 2)
    one = _run(w, Y, tr, te, "16")
    many = _run(w, Y, tr, te, "0.011")  # about 11 MB of scratch per chunk: four or five chunks
    for k in ("mixed", "fp32", "grid"):
        assert np.linalg.norm(many[k] - one[k]) <= 1e-12 * np.linalg.norm(one[k]), k
    np.testing.assert_array_equal(many["best"], one["best"])
