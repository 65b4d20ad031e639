"""The N-GPU bench path on the CPU: two gloo ranks (world size 2) through bench.py's own code.

bench.py --gpus N shards one hemisphere over the N ranks (bench.sharded_rank: contiguous
searchlight ranges, column owners, one all-to-all of partial CSC values per step) and keeps N
independent replicas as a sub-field.  Here the ranks run that rank code with partial values from
the oracle: the assembled result must equal the same split combined in one process bit for bit
and the whole hemisphere up to the association of the float64 sums; the job time is the max over
ranks and the replica value the whole-job aggregate.
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


def _sharded_main(rank, ws, port, out, case):
    sys.path.insert(0, ROOT)
    import datetime
    import torch
    import torch.distributed as dist
    import bench
    from hyperalignment_b200 import shard as S
    from oracle import ha_oracle as O
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    w, wts, T = case

    def partial_np(lo, hi):
        idx, off, sw = S.sub_geometry(w.sls.indices, w.sls.offsets, wts, lo, hi)
        indptr, rows = O.sparse_init(idx, off, w.nv)
        data = np.zeros(rows.size)
        O.searchlight_procrustes_csc(w.X, w.Y, idx, off, indptr, rows, data, weights=sw, transforms=T[lo:hi])
        return indptr.astype(np.int64), rows, data

    def make_range(lo, hi):
        indptr, rows, data = partial_np(lo, hi)
        src = torch.from_numpy(data)
        return indptr, rows, lambda partial: partial.copy_(src)

    res = bench.sharded_rank(ws, rank, w.sls.offsets, w.nv, make_range, 3, 1, "cpu")
    full = res["exchange"].assemble(res["owned"], dst=0)
    if rank == 0:
        same = bench.sharded_same_split(w.sls.offsets, w.nv, ws,
                                        lambda lo, hi: (lambda p: (p[0], p[1], torch.from_numpy(p[2])))(partial_np(lo, hi)))
        np.savez(os.path.join(out, "sharded.npz"), indptr=full[0], rows=full[1], vals=full[2],
                 bitwise=bench.bitwise_equal(full, same), job=res["job_ms"], solve=res["solve_ms"],
                 exch=res["exchange_ms"], bounds=res["bounds"])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_hemisphere(tmp_path):
    """bench.py --gpus 2's rank code (bench.sharded_rank) over two gloo ranks."""
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_shard import _case, _full
    w, wts, T = _case(seed=9)
    mp.spawn(_sharded_main, args=(2, _free_port(), str(tmp_path), (w, wts, T)), nprocs=2, join=True)
    r = np.load(tmp_path / "sharded.npz")
    indptr, rows, data = _full(w, wts, T)
    assert bool(r["bitwise"])                                   # same split in one process: identical bits
    assert np.array_equal(r["indptr"], indptr) and np.array_equal(r["rows"], rows)
    assert np.linalg.norm(r["vals"] - data) <= 1e-13 * np.linalg.norm(data)
    assert 0 < r["bounds"][1] < w.sls.count                     # both ranks hold searchlights
    assert r["job"] >= r["solve"] and r["job"] >= r["exch"] >= 0.0

