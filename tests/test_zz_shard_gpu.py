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


def test_bench_sharded_path_one_rank_nccl(gpu, capsys):
    """bench.py --gpus N's sharded rank code (bench.run_sharded_b200) on a one-rank NCCL group: the
    same collectives (all-reduce, all-to-all, point-to-point assembly) on this GPU alone, and the
    line's own checks: bit-identical to the same split solved on rank 0, the one plan's pattern."""
    import argparse
    import json
    import os
    import socket
    import sys
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=120))
    args = argparse.Namespace(nv=2562, nt=200, steps=2, warmup=1)
    bench.run_sharded_b200(args, 1, 0, 0, L.lib())
    assert not dist.is_initialized()
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["n_gpus"] == 1 and line["scaling"] == "strong" and line["value"] > 0
    assert line["exchange_ms_per_step"] >= 0.0 and line["solve_ms_per_step"] > 0.0
    chk = line["vs_one_plan"]
    assert chk["bitwise_vs_same_split_on_rank0"] and chk["pattern_identical_to_one_plan"]
    assert chk["values_relfrob_vs_one_plan"] <= 1e-12
    assert line["replicas"]["value"] > 0 and line["e2e"]["value"] > 0
