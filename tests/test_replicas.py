"""The N-GPU bench path on the CPU: two gloo ranks (world size 2) through bench.py's own helpers.

bench.py --gpus N runs N independent replicas (one subject pair per rank, no data-path exchange).
What the ranks share is the timing: the job time is the max over ranks and the value is the
whole-job aggregate.  This checks those helpers across real processes, and that the replicas
solve different inputs.
"""

import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    wsz, r, local = bench.dist_setup(None)
    local_ms = 100.0 + 50.0 * rank               # rank 1 is the slower one
    job_ms = bench.max_over_ranks(local_ms, wsz)
    rate = bench.aggregate_rate(wsz, 1000, 3, job_ms / 1e3)
    w = bench.workload(r, 162, 20)  # the replica's subject pair (seed = rank)
    sig = float(w.X[:4, :4].sum())
    dist.barrier()
    dist.destroy_process_group()
    np.save(os.path.join(out, f"r{rank}.npy"), np.array([wsz, r, job_ms, rate, sig]))


def test_two_rank_timing_and_replicas(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r0 = np.load(tmp_path / "r0.npy")
    r1 = np.load(tmp_path / "r1.npy")
    assert r0[0] == 2 and r1[0] == 2 and (r0[1], r1[1]) == (0, 1)
    assert r0[2] == r1[2] == 150.0                      # job time = max over ranks
    assert r0[3] == pytest.approx(2 * 1000 * 3 / 0.150)  # whole-job aggregate
    assert r0[4] != r1[4]                               # each replica solves its own subject pair
