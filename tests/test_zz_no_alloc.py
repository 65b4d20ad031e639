"""The allocation-free entry point ha_b200_local_procrustes_noalloc, through the C ABI.

Callers that cannot allocate device memory (their pool allocator owns the GPU, their host
program forbids new allocations, or cudaMalloc's device-wide synchronisation is not acceptable
in their loop) pass their own device buffers and the library uses only a static scratch array.
Its output must match the allocating plan API's plain FP32 local transforms on the same inputs,
within the per-transform tolerance of the parity tests, on two calls in a row (the shared scratch
keeps the previous call's contents).  The inputs have more samples than any searchlight has
vertices, so every transform is unique and two correct solvers agree.  The file sorts after the
parity tests so that a run stopping at the first failure has run them first.
"""

import ctypes

import numpy as np
import pytest

from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import workloads as W
from hyperalignment_b200.plan import Plan

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


def test_noalloc_matches_plan_on_two_calls(gpu):
    import torch
    w = W.small_case(seed=31, nv=642, nt=400, lo=1, hi=160)
    s = w.sls
    d_idx = torch.from_numpy(s.indices).cuda()
    total = int((s.sizes.astype(np.int64) ** 2).sum())
    for X, Y in ((w.X, w.Y), (w.Y, w.X)):
        ref = _plan_transforms(w, X, Y)
        dX = torch.from_numpy(np.asfortranarray(X).ravel(order="F")).cuda()
        dY = torch.from_numpy(np.asfortranarray(Y).ravel(order="F")).cuda()
        out = torch.full((total,), float("nan"), dtype=torch.float32, device="cuda")
        rc = gpu.ha_b200_local_procrustes_noalloc(ctypes.c_void_p(dX.data_ptr()), ctypes.c_void_p(dY.data_ptr()),
                                                  w.nt, w.nv, ctypes.c_void_p(d_idx.data_ptr()), L.iptr(s.offsets),
                                                  s.count, ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0
        got = out.cpu().numpy().astype(np.float64)
        o = 0
        worst = 0.0
        for q in range(s.count):
            n = int(s.sizes[q])
            T = got[o:o + n * n].reshape(n, n)
            o += n * n
            worst = max(worst, float(np.linalg.norm(T - ref[q]) / np.linalg.norm(ref[q])))
        assert worst <= TOL, worst


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
