"""One hemisphere sharded over ranks, the GPU side, emulated in one process on one GPU.

Each emulated rank builds a plan of its searchlight range with the hemisphere's weights and
solves it on the GPU, as ShardedSearchlights does on its own GPU. The exchange then runs in
process (shard.exchange_in_process), with no collective and no kernel that waits on another. The
result must have the whole hemisphere's pattern exactly, and the one-plan values up to the order
of the float64 additions. The per-searchlight transforms do not depend on which plan solved them.
The file sorts after the other GPU tests, so a run stopping at the first failure has run them
first.
"""

import numpy as np
import pytest

from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import shard as S
from hyperalignment_b200 import workloads as W
from hyperalignment_b200.plan import Plan

pytestmark = pytest.mark.gpu

REL = {L.SOLVER_FP64: 1e-10, L.SOLVER_MIXED: 1e-5}  # relative Frobenius vs the one-plan result


def _solve(plan, dX, dY, solver):
    import torch
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
    plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, True, solver, L.OUT_CSC)
    torch.cuda.synchronize()
    return vals


@pytest.mark.parametrize("solver", [L.SOLVER_FP64, L.SOLVER_MIXED])
def test_sharded_plans_equal_one_plan(gpu, solver):
    import torch
    w = W.small_case(seed=5, nv=2562, nt=160, lo=40, hi=100, scaling=True)
    s = w.sls
    wts = S.hemisphere_weights(s.indices, s.offsets, s.dists, s.radius, w.nv)
    dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).cuda()
    dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).cuda()
    whole = Plan(w.nt, w.nv, s.indices, s.offsets, weights=wts)
    indptr, rows = whole.pattern()
    ref = _solve(whole, dX, dY, solver).cpu().numpy()
    whole.close()
    for world in (2, 3):
        b = S.split_searchlights(s.offsets, world)
        ptrs, rws, parts = [], [], []
        for r in range(world):
            idx, off, sw = S.sub_geometry(s.indices, s.offsets, wts, int(b[r]), int(b[r + 1]))
            plan = Plan(w.nt, w.nv, idx, off, weights=sw)
            p, q = plan.pattern()
            ptrs.append(p)
            rws.append(q)
            parts.append(_solve(plan, dX, dY, solver))
            plan.close()
        got = S.exchange_in_process(ptrs, rws, parts, w.nv)
        np.testing.assert_array_equal(got[0], indptr)
        np.testing.assert_array_equal(got[1], rows)
        rel = np.linalg.norm(got[2] - ref) / np.linalg.norm(ref)
        assert rel <= REL[solver], (world, rel)
