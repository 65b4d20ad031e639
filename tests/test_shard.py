"""One hemisphere sharded over ranks (hyperalignment_b200/shard.py), on the CPU.

The partial values of each rank come from the oracle here: the searchlight Procrustes of the
rank's searchlights with the hemisphere's weights, scattered into the rank's own CSC pattern. The
exchange must give the reference's pattern of the whole hemisphere exactly
(csrc/ha_sparse.c:31-112) and the sum over all searchlights (csrc/ha_searchlight.c:147-201) up to
the order of the float64 additions. It is checked in one process for several world sizes, and
across two and three gloo ranks through torch.distributed.
"""

import os
import socket
import sys

import numpy as np
import pytest

from hyperalignment_b200 import shard as S
from hyperalignment_b200 import workloads as W
from oracle import ha_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-13  # relative Frobenius: only the association of the float64 sums differs


def _case(seed=7):
    w = W.small_case(seed=seed, nv=642, nt=40, lo=20, hi=60, scaling=True)
    sls = w.sls
    wts = S.hemisphere_weights(sls.indices, sls.offsets, sls.dists, sls.radius, w.nv)
    T = O.local_transforms(w.X, w.Y, sls.indices, sls.offsets, w.reflection, w.scaling)
    return w, wts, T


def _full(w, wts, T):
    indptr, rows = O.sparse_init(w.sls.indices, w.sls.offsets, w.nv)
    data = np.zeros(rows.size)
    O.searchlight_procrustes_csc(w.X, w.Y, w.sls.indices, w.sls.offsets, indptr, rows, data, weights=wts,
                                 transforms=T)
    return indptr.astype(np.int64), rows, data


def _partial(w, wts, T, lo, hi):
    """Rank pattern and partial values for searchlights [lo, hi) (empty when lo == hi)."""
    if hi == lo:
        return np.zeros(w.nv + 1, dtype=np.int64), np.zeros(0, dtype=np.int32), np.zeros(0)
    idx, off, sw = S.sub_geometry(w.sls.indices, w.sls.offsets, wts, lo, hi)
    indptr, rows = O.sparse_init(idx, off, w.nv)
    data = np.zeros(rows.size)
    O.searchlight_procrustes_csc(w.X, w.Y, idx, off, indptr, rows, data, weights=sw, transforms=T[lo:hi])
    return indptr.astype(np.int64), rows, data


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_hemisphere_weights_match_oracle():
    w = W.small_case(seed=2, nv=642, nt=40, lo=20, hi=60)
    s = w.sls
    ours = S.hemisphere_weights(s.indices, s.offsets, s.dists, s.radius, w.nv)
    assert np.array_equal(ours, O.searchlight_weights(s.indices, s.offsets, s.dists, s.radius, w.nv))
    uni = S.hemisphere_weights(s.indices, s.offsets, None, 0.0, w.nv)
    assert np.array_equal(uni, O.searchlight_weights(s.indices, s.offsets, None, 0.0, w.nv))


def test_split_searchlights_balanced_and_contiguous():
    rng = np.random.default_rng(0)
    sizes = rng.integers(50, 501, size=4000)
    off = np.concatenate([[0], np.cumsum(sizes)])
    cost = sizes.astype(np.float64) ** 3
    for world in (1, 2, 3, 8):
        b = S.split_searchlights(off, world)
        assert b[0] == 0 and b[-1] == sizes.size and np.all(np.diff(b) >= 0)
        share = np.array([cost[b[r]:b[r + 1]].sum() for r in range(world)]) / cost.sum()
        assert np.all(np.abs(share - 1.0 / world) <= 501.0 ** 3 / cost.sum())  # off by one searchlight at most
    b = S.split_searchlights(off[:4], 8)  # fewer searchlights than ranks: some ranks get none
    assert b[0] == 0 and b[-1] == 3 and np.all(np.diff(b) >= 0)


def test_split_columns_balanced():
    rng = np.random.default_rng(1)
    counts = rng.integers(0, 300, size=10242)
    for world in (1, 2, 4, 8):
        c = S.split_columns(counts, world)
        assert c[0] == 0 and c[-1] == counts.size and np.all(np.diff(c) >= 0)
        share = np.array([counts[c[q]:c[q + 1]].sum() for q in range(world)])
        assert np.all(np.abs(share - counts.sum() / world) <= counts.max())
    assert np.array_equal(S.split_columns(np.zeros(5, np.int64), 2), [0, 0, 5])


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_exchange_in_process_equals_whole_hemisphere(world):
    import torch
    w, wts, T = _case()
    indptr, rows, data = _full(w, wts, T)
    b = S.split_searchlights(w.sls.offsets, world)
    parts = [_partial(w, wts, T, int(b[r]), int(b[r + 1])) for r in range(world)]
    got = S.exchange_in_process([p[0] for p in parts], [p[1] for p in parts],
                                [torch.from_numpy(p[2]) for p in parts], w.nv)
    assert np.array_equal(got[0], indptr)
    assert np.array_equal(got[1], rows)
    assert _rel(got[2], data) <= TOL
    again = S.exchange_in_process([p[0] for p in parts], [p[1] for p in parts],
                                  [torch.from_numpy(p[2]) for p in parts], w.nv)
    assert np.array_equal(again[2], got[2])  # deterministic


def test_exchange_with_an_empty_rank():
    import torch
    w, wts, T = _case(seed=3)
    indptr, rows, data = _full(w, wts, T)
    n = w.sls.count
    cuts = [(0, n // 2), (n // 2, n // 2), (n // 2, n)]  # rank 1 solves nothing
    parts = [_partial(w, wts, T, lo, hi) for lo, hi in cuts]
    got = S.exchange_in_process([p[0] for p in parts], [p[1] for p in parts],
                                [torch.from_numpy(p[2]) for p in parts], w.nv)
    assert np.array_equal(got[0], indptr) and np.array_equal(got[1], rows)
    assert _rel(got[2], data) <= TOL


def test_column_exchange_single_process():
    """No process group: the one process owns every column and nothing is exchanged."""
    import torch
    import torch.distributed as dist
    assert not dist.is_initialized()
    w, wts, T = _case()
    indptr, rows, data = _full(w, wts, T)
    ex = S.ColumnExchange(indptr, rows, w.nv)
    assert ex.world == 1 and ex.col_range == (0, w.nv)
    owned = ex.combine(torch.from_numpy(data))
    got = ex.assemble(owned)
    assert np.array_equal(got[0], indptr) and np.array_equal(got[1], rows)
    assert np.array_equal(got[2], data)
    with pytest.raises(ValueError):
        S.ColumnExchange(indptr[:-1], rows, w.nv)
    with pytest.raises(ValueError):
        S.ColumnExchange(indptr, rows[:-1], w.nv)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange(w, wts, T, group, out, tag):
    import torch.distributed as dist
    import torch
    from hyperalignment_b200 import shard
    ws, rank = dist.get_world_size(group), dist.get_rank(group)
    b = shard.split_searchlights(w.sls.offsets, ws)
    indptr, rows, part = _partial(w, wts, T, int(b[rank]), int(b[rank + 1]))
    ex = shard.ColumnExchange(indptr, rows, w.nv, group=group)
    owned = ex.combine(torch.from_numpy(part))
    lo, hi = ex.col_range
    res = ex.assemble(owned, dst=0)
    np.savez(os.path.join(out, f"{tag}_r{rank}.npz"), lo=lo, hi=hi, owned=owned.numpy(),
             **({} if res is None else {"indptr": res[0], "rows": res[1], "vals": res[2]}))


def _rank_main(rank, ws, port, out, case):
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    w, wts, T = case  # made once by the parent (BLAS threads of three ranks at once oversubscribe the host)
    _exchange(w, wts, T, None, out, f"w{ws}")          # every rank
    pair = dist.new_group([1, 2])                       # every rank takes part in creating it
    if rank >= 1:
        _exchange(w, wts, T, pair, out, "w2")           # world size 2, group ranks != global ranks
    dist.barrier()
    dist.destroy_process_group()


def test_column_exchange_over_gloo(tmp_path):
    import torch.multiprocessing as mp
    w, wts, T = _case()
    mp.spawn(_rank_main, args=(3, _free_port(), str(tmp_path), (w, wts, T)), nprocs=3, join=True)
    indptr, rows, data = _full(w, wts, T)
    for world in (3, 2):
        r = [np.load(tmp_path / f"w{world}_r{q}.npz") for q in range(world)]
        assert r[0]["lo"] == 0 and r[-1]["hi"] == w.nv
        assert all(r[q]["hi"] == r[q + 1]["lo"] for q in range(world - 1))
        for q in range(world):  # each owner holds exactly its columns' values
            lo, hi = int(r[q]["lo"]), int(r[q]["hi"])
            assert _rel(r[q]["owned"], data[indptr[lo]:indptr[hi]]) <= TOL
        assert np.array_equal(r[0]["indptr"], indptr)
        assert np.array_equal(r[0]["rows"], rows)
        assert _rel(r[0]["vals"], data) <= TOL
