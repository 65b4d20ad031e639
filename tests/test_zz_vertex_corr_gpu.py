"""Vertex-wise correlation of aligned data with the target (ha_b200_aligned_correlation_device).

The evaluation step of the reference's benchmark (benchmark_neuroboros.py:204-211 and :229-232):
the searchlight Procrustes W of a subject pair fitted on training time points, A = X_test @ W,
and per vertex the mean over time of zscore(A) * zscore(Y_test). It is compared with the oracle
on the same W (the plan's CSC values). The unaligned correlation (no W) is checked too, and a
constant target column must give NaN in both. The file sorts after the other GPU tests, so a run
stopping at the first failure has run them first.
"""

import numpy as np
import pytest

from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import workloads as W
from hyperalignment_b200.plan import Plan
from oracle import ha_oracle as O

pytestmark = pytest.mark.gpu

ATOL = 1e-12  # on r, float64 on both sides; only the summation order differs


def _dev(M):
    import torch
    return torch.from_numpy(np.asfortranarray(M).ravel(order="F")).cuda()


def test_vertex_correlation_matches_oracle(gpu):
    import scipy.sparse as sp
    import torch
    w = W.small_case(seed=9, nv=642, nt=120, lo=20, hi=60, scaling=True)
    s = w.sls
    n_fit = 80
    Xtr, Ytr, Xte, Yte = w.X[:n_fit], w.Y[:n_fit], w.X[n_fit:], w.Y[n_fit:]
    nte = Xte.shape[0]
    plan = Plan(n_fit, w.nv, s.indices, s.offsets, s.dists, s.radius)
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
    dXtr, dYtr = _dev(Xtr), _dev(Ytr)  # held: the library reads them after the call returns
    plan.procrustes_device(dXtr.data_ptr(), dYtr.data_ptr(), vals.data_ptr(), True, True, L.SOLVER_MIXED, L.OUT_CSC)
    torch.cuda.synchronize()
    indptr, rows = plan.pattern()
    Wm = sp.csc_matrix((vals.cpu().numpy(), rows, indptr), shape=(w.nv, w.nv))

    dXte, dYte = _dev(Xte), _dev(Yte)
    r = torch.zeros(w.nv, dtype=torch.float64, device="cuda")
    A = torch.zeros(nte * w.nv, dtype=torch.float64, device="cuda")
    plan.aligned_correlation_device(dXte.data_ptr(), dYte.data_ptr(), vals.data_ptr(), r.data_ptr(), A.data_ptr(),
                                    nt=nte)
    torch.cuda.synchronize()
    r_ref = O.aligned_correlation(Xte, Yte, Wm)
    assert np.isfinite(r_ref).all()
    assert np.abs(r.cpu().numpy() - r_ref).max() <= ATOL
    A_ref = np.asarray(Xte @ Wm)
    A_got = A.cpu().numpy().reshape(w.nv, nte).T
    assert np.linalg.norm(A_got - A_ref) <= 1e-13 * np.linalg.norm(A_ref)

    # without the aligned buffer the second pass recomputes A in the same order: identical r
    r2 = torch.zeros_like(r)
    plan.aligned_correlation_device(dXte.data_ptr(), dYte.data_ptr(), vals.data_ptr(), r2.data_ptr(), nt=nte)
    torch.cuda.synchronize()
    assert torch.equal(r2, r)

    # the unaligned correlation (W = identity), as the reference's r_test0
    r0 = torch.zeros_like(r)
    plan.aligned_correlation_device(dXte.data_ptr(), dYte.data_ptr(), 0, r0.data_ptr(), nt=nte)
    torch.cuda.synchronize()
    assert np.abs(r0.cpu().numpy() - O.aligned_correlation(Xte, Yte)).max() <= ATOL

    # the fit is real: alignment raises the mean correlation on the held-out time points
    assert float(r.mean()) > float(r0.mean()) + 0.05

    # a constant target column: NaN, as scipy's z-score gives
    Yc = Yte.copy()
    Yc[:, 5] = 1.5
    rc = torch.zeros_like(r)
    dYc = _dev(Yc)
    plan.aligned_correlation_device(dXte.data_ptr(), dYc.data_ptr(), vals.data_ptr(), rc.data_ptr(), nt=nte)
    torch.cuda.synchronize()
    got = rc.cpu().numpy()
    want = O.aligned_correlation(Xte, Yc, Wm)
    assert np.isnan(got[5]) and np.isnan(want[5])
    assert np.abs(np.delete(got, 5) - np.delete(want, 5)).max() <= ATOL
    plan.close()
