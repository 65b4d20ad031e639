"""The allocation-free entry point ha_b200_local_procrustes_noalloc, through the C ABI.

Callers that cannot allocate device memory (their pool allocator owns the GPU, their host
program forbids new allocations, or cudaMalloc's device-wide synchronisation is not acceptable
in their loop) pass their own device buffers and the library uses only a static scratch array.
Its output must match the allocating plan API's plain FP32 local transforms on the same inputs,
within the per-transform tolerance of the parity tests, on two calls in a row (the shared scratch
keeps the previous call's contents), and the float64 oracle directly.  The inputs have more
samples than any searchlight has vertices, so every transform is unique and two correct solvers
agree.  The file sorts after the parity tests so that a run stopping at the first failure has
run them first.
"""

import ctypes

import numpy as np
import pytest

from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import workloads as W
from hyperalignment_b200.plan import Plan
from oracle import ha_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-4  # relative Frobenius per transform, as in the parity tests


def _plan_transforms(w, X, Y):
    import torch
    plan = Plan(w.nt, w.nv, w.sls.indices, w.sls.offsets, w.sls.dists, w.sls.radius)
    dX = torch.from_numpy(np.asfortranarray(X).ravel(order="F")).cuda()
    dY = torch.from_numpy(np.asfortranarray(Y).ravel(order="F")).cuda()
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
    plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, False, L.SOLVER_FP32, L.OUT_CSR)
    torch.cuda.synchronize()
    Ts = plan.local_transforms(0, w.sls.count)
    plan.close()
    return Ts


def _noalloc(lib, w, X, Y, indices=None):
    """One call; returns (return code, the packed transforms as a list of n x n arrays)."""
    import torch
    s = w.sls
    idx = s.indices if indices is None else indices
    d_idx = torch.from_numpy(np.ascontiguousarray(idx, dtype=np.int32)).cuda()
    total = int((s.sizes.astype(np.int64) ** 2).sum())
    dX = torch.from_numpy(np.asfortranarray(X).ravel(order="F")).cuda()
    dY = torch.from_numpy(np.asfortranarray(Y).ravel(order="F")).cuda()
    out = torch.full((total,), float("nan"), dtype=torch.float32, device="cuda")
    rc = lib.ha_b200_local_procrustes_noalloc(ctypes.c_void_p(dX.data_ptr()), ctypes.c_void_p(dY.data_ptr()),
                                              w.nt, w.nv, ctypes.c_void_p(d_idx.data_ptr()), L.iptr(s.offsets),
                                              s.count, ctypes.c_void_p(out.data_ptr()), None)
    got = out.cpu().numpy().astype(np.float64)
    Ts, o = [], 0
    for q in range(s.count):
        n = int(s.sizes[q])
        Ts.append(got[o:o + n * n].reshape(n, n))
        o += n * n
    return rc, Ts


def _worst(Ts, refs):
    return max(float(np.linalg.norm(T - R) / np.linalg.norm(R)) for T, R in zip(Ts, refs))


def test_noalloc_matches_plan_on_two_calls(gpu):
    w = W.small_case(seed=31, nv=642, nt=400, lo=1, hi=160)
    for X, Y in ((w.X, w.Y), (w.Y, w.X)):
        rc, Ts = _noalloc(gpu, w, X, Y)
        assert rc == 0
        assert _worst(Ts, _plan_transforms(w, X, Y)) <= TOL


def test_noalloc_matches_oracle(gpu):
    """Against the float64 restatement of the reference's local Procrustes directly."""
    w = W.small_case(seed=33, nv=642, nt=300, lo=5, hi=160)
    rc, Ts = _noalloc(gpu, w, w.X, w.Y)
    assert rc == 0
    s = w.sls
    pick = np.arange(0, s.count, 7)
    refs = [O.procrustes(w.X[:, s.indices[s.offsets[q]:s.offsets[q + 1]]],
                         w.Y[:, s.indices[s.offsets[q]:s.offsets[q + 1]]]) for q in pick]
    assert _worst([Ts[q] for q in pick], refs) <= TOL


@pytest.mark.parametrize("nv,lo,hi", [(2562, 1, 12),      # 2562 items: more than one 2048-item batch
                                      (1442, 150, 160)])  # large matrices: the scratch area splits batches
def test_noalloc_several_batches(gpu, nv, lo, hi):
    """Work split over several batches (output offsets carried between them), twice in a row.
    Compared with the plan on the searchlights FP32 resolves (sigma_min / sigma_max >= 1e-4): below
    that the plan's blocked FP32 Jacobi and this entry's resident one round differently and may
    settle the smallest singular direction differently (the plain FP32 form's known limit); every
    transform must still be orthogonal."""
    w = W.small_case(seed=35, nv=nv, nt=max(2 * hi, 40), lo=lo, hi=hi)
    s = w.sls
    ratio = np.array([(lambda v: v[-1] / v[0])(np.linalg.svd(
        w.X[:, s.indices[s.offsets[q]:s.offsets[q + 1]]].T @ w.Y[:, s.indices[s.offsets[q]:s.offsets[q + 1]]],
        compute_uv=False)) for q in range(s.count)])
    keep = np.flatnonzero(ratio >= 1e-4)
    assert keep.size >= s.count // 2
    ref = _plan_transforms(w, w.X, w.Y)
    for _ in range(2):
        rc, Ts = _noalloc(gpu, w, w.X, w.Y)
        assert rc == 0
        assert _worst([Ts[q] for q in keep], [ref[q] for q in keep]) <= TOL
        assert max(float(np.abs(T.T @ T - np.eye(T.shape[0])).max()) for T in Ts) < 1e-4


def test_noalloc_rejects_out_of_range_index(gpu):
    """A vertex index equal to nv is caught by the kernel's own check (read as a zero column, never
    dereferenced) and reported as an argument error; the next call succeeds."""
    w = W.small_case(seed=37, nv=162, nt=40, lo=8, hi=24)
    bad = w.sls.indices.copy()
    bad[len(bad) // 2] = w.nv
    rc, _ = _noalloc(gpu, w, w.X, w.Y, indices=bad)
    assert rc == L.ERROR_ARG
    rc, Ts = _noalloc(gpu, w, w.X, w.Y)
    assert rc == 0
    assert _worst(Ts, _plan_transforms(w, w.X, w.Y)) <= TOL


def test_noalloc_rejects_oversized_searchlights(gpu):
    import torch
    nt, nv = 8, 200
    d = torch.zeros(nt * nv, dtype=torch.float64, device="cuda")
    idx = torch.arange(nv, dtype=torch.int32, device="cuda")
    off = np.array([0, 161], dtype=np.int32)
    out = torch.zeros(161 * 161, dtype=torch.float32, device="cuda")
    rc = gpu.ha_b200_local_procrustes_noalloc(ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()), nt, nv,
                                              ctypes.c_void_p(idx.data_ptr()), L.iptr(off), 1,
                                              ctypes.c_void_p(out.data_ptr()), None)
    assert rc == L.ERROR_ARG
