"""One hemisphere's searchlight solves sharded over ranks, one process per GPU.

The reference solves every searchlight of a hemisphere in one OpenMP loop and adds each weighted
local transform into the one shared result (csrc/ha_searchlight.c:147-201 with
csrc/ha_sparse.c:128-142 for the CSC matrix, csrc/ha_searchlight.c:1073-1099 for the dense one).
Sharded here:

* Searchlights are split into contiguous ranges, one per rank, balanced by the sum of n^3 (the
  cost of a local solve). Each rank solves its range on its own GPU with the weights of the whole
  hemisphere (csrc/ha_searchlight.c:970-1001 sums them over every searchlight), which gives
  partial CSC values over the pattern of its own searchlights.
* Every CSC column has one owner rank: contiguous column ranges balanced by the summed pattern
  sizes. Once per geometry the ranks send each owner the row lists of its columns. The owner
  builds the union pattern of its columns, which is the reference's pattern restricted to them
  (csrc/ha_sparse.c:31-112), and records where each source's entries land in it.
* Per solve, one variable-size all-to-all carries the partial values to the owners, and each
  owner adds the sources' partials in rank order. The result is deterministic for a given world
  size. It equals the one-GPU result up to the order of the float64 additions.

The partial values come from the library (``ha_b200_plan_procrustes_device`` on a plan of the
rank's searchlights). torch.distributed moves them (NCCL between GPUs, gloo on the CPU) and torch
indexes them into place. The pieces that need no collective (`split_searchlights`,
`split_columns`, `owner_map`, `combine`) are plain functions, so one process can also run the
whole exchange for every rank.
"""

from __future__ import annotations

import dataclasses

import numpy as np

from . import _lib as L


def split_searchlights(offsets, world: int) -> np.ndarray:
    """Boundaries b (world + 1 entries): rank r solves searchlights [b[r], b[r+1]), contiguous
    ranges balanced by the sum of n^3 over their searchlights."""
    off = np.asarray(offsets, dtype=np.int64)
    count = off.size - 1
    cost = np.diff(off).astype(np.float64) ** 3
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    b = np.searchsorted(cum, cum[-1] * np.arange(world + 1) / world, side="left")
    b[0], b[-1] = 0, count
    return np.maximum.accumulate(np.minimum(b, count)).astype(np.int64)


def split_columns(col_counts, world: int) -> np.ndarray:
    """Boundaries c (world + 1 entries): rank q owns CSC columns [c[q], c[q+1]), contiguous ranges
    balanced by the pattern entries per column."""
    counts = np.asarray(col_counts, dtype=np.int64)
    nv = counts.size
    cum = np.concatenate([[0], np.cumsum(counts)])
    c = np.searchsorted(cum, cum[-1] * np.arange(world + 1) / world, side="left")
    c[0], c[-1] = 0, nv
    return np.maximum.accumulate(np.minimum(c, nv)).astype(np.int64)


def sub_geometry(indices, offsets, weights, lo: int, hi: int):
    """Flat indices, rebased offsets and weights of searchlights [lo, hi)."""
    a, b = int(offsets[lo]), int(offsets[hi])
    idx = np.ascontiguousarray(indices[a:b], dtype=np.int32)
    off = np.ascontiguousarray(np.asarray(offsets[lo:hi + 1], dtype=np.int64) - a, dtype=np.int32)
    return idx, off, np.ascontiguousarray(weights[a:b], dtype=np.float64)


def hemisphere_weights(indices, offsets, dists, radius: float, nv: int) -> np.ndarray:
    """Flat weights over the whole hemisphere, computed by the library on the host with the
    reference's operation order (csrc/ha_searchlight.c:970-1001); uniform when dists is None."""
    idx = np.ascontiguousarray(indices, dtype=np.int32)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    d = None if dists is None else np.ascontiguousarray(dists, dtype=np.float64)
    out = np.empty(idx.size, dtype=np.float64)
    L.check(L.lib().ha_searchlight_weights_b200(L.iptr(idx), L.iptr(off), L.dptr(d), off.size - 1,
                                                float(radius or 0.0), int(nv), L.dptr(out)),
            "ha_searchlight_weights_b200")
    return out


@dataclasses.dataclass
class OwnerMap:
    """The owner's side of the exchange for columns [col_lo, col_hi)."""
    col_lo: int
    col_hi: int
    indptr: object      # int64, (col_hi - col_lo + 1), relative to the first owned entry
    indices: object     # int32 rows of the owned columns, ascending within each column
    positions: list     # per source rank: int64 positions of its entries in the owned values

    @property
    def nnz(self) -> int:
        return int(self.indices.numel())


def owner_map(nv: int, col_lo: int, col_hi: int, counts_in: list, rows_in: list) -> OwnerMap:
    """Union pattern of the owned columns and every source's positions in it.

    counts_in[s]: entries per owned column in source s's pattern (col_hi - col_lo values);
    rows_in[s]: those entries' rows, column by column, ascending within a column (CSC order)."""
    import torch
    ncols = col_hi - col_lo
    keys = []
    for cnt, rows in zip(counts_in, rows_in):
        col = torch.repeat_interleave(torch.arange(ncols, device=cnt.device, dtype=torch.int64), cnt.to(torch.int64))
        keys.append(col * nv + rows.to(torch.int64))
    every = torch.cat(keys) if keys else torch.zeros(0, dtype=torch.int64)
    owned = torch.unique(every, sorted=True)
    col = owned // nv
    indptr = torch.zeros(ncols + 1, dtype=torch.int64, device=owned.device)
    indptr[1:] = torch.cumsum(torch.bincount(col, minlength=ncols), 0)
    positions = [torch.searchsorted(owned, k) for k in keys]
    return OwnerMap(col_lo, col_hi, indptr, (owned - col * nv).to(torch.int32), positions)


def combine(omap: OwnerMap, values_in: list):
    """Owned values: 0 plus every source's partial values, added in rank order. Within one source
    the positions are distinct, so the result does not depend on how the adds are scheduled."""
    import torch
    dev = omap.indices.device
    out = torch.zeros(omap.nnz, dtype=torch.float64, device=dev)
    for pos, vals in zip(omap.positions, values_in):
        if pos.numel():
            out.index_add_(0, pos, vals)
    return out


def exchange_in_process(indptrs: list, rows: list, partials: list, nv: int):
    """The whole exchange for every rank inside one process (no collective): rank s's pattern is
    (indptrs[s], rows[s]) and its partial values partials[s] (torch, CSC order). Returns the
    assembled matrix (indptr int64, indices int32, values float64, numpy) as the owners would
    hold it, column ranges from `split_columns` as in `ColumnExchange`."""
    import torch
    world = len(indptrs)
    lps = [np.asarray(p, dtype=np.int64) for p in indptrs]
    c = split_columns(sum(np.diff(p) for p in lps), world)
    out_ptr = np.zeros(nv + 1, dtype=np.int64)
    out_rows, out_vals, base = [], [], 0
    for q in range(world):
        lo, hi = int(c[q]), int(c[q + 1])
        counts_in, rows_in, vals_in = [], [], []
        for s in range(world):
            a, b = int(lps[s][lo]), int(lps[s][hi])
            counts_in.append(torch.from_numpy(np.diff(lps[s][lo:hi + 1])).to(partials[s].device))
            rows_in.append(torch.as_tensor(np.asarray(rows[s][a:b], dtype=np.int32)).to(partials[s].device))
            vals_in.append(partials[s][a:b])
        omap = owner_map(nv, lo, hi, counts_in, rows_in)
        vals = combine(omap, vals_in)
        out_ptr[lo + 1:hi + 1] = base + omap.indptr[1:].cpu().numpy()
        base += omap.nnz
        out_rows.append(omap.indices.cpu().numpy())
        out_vals.append(vals.cpu().numpy())
    return out_ptr, np.concatenate(out_rows), np.concatenate(out_vals)


def _world_rank(group):
    """(world size, rank) of the group; (1, 0) without a group when no process group is up."""
    import torch.distributed as dist
    if group is None and not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def _global(group, q):
    """Global rank of the group's rank q (point-to-point calls take global ranks)."""
    import torch.distributed as dist
    return q if group is None else dist.get_global_rank(group, q)


class ColumnExchange:
    """The exchange between a rank's pattern and the column owners over a torch.distributed
    group: built once per geometry (two all-to-alls of the row lists), then one all-to-all of
    float64 values per solve. Without a group and with no process group initialised, the one
    process owns every column and nothing is exchanged."""

    def __init__(self, indptr, indices, nv: int, group=None, device="cpu"):
        import torch
        import torch.distributed as dist
        self.group = group
        self.single = group is None and not dist.is_initialized()
        self.world, self.rank = _world_rank(group)
        self.nv = int(nv)
        lp = np.asarray(indptr, dtype=np.int64)
        if lp.size != self.nv + 1 or lp[0] != 0 or np.any(np.diff(lp) < 0):
            raise ValueError("indptr must be a CSC column pointer of nv + 1 non-decreasing entries from 0")
        counts = torch.from_numpy(np.diff(lp)).to(device)
        rows = torch.as_tensor(np.asarray(indices, dtype=np.int32)).to(device)
        if rows.numel() != int(lp[-1]):
            raise ValueError("indices must hold indptr[nv] rows")
        if self.single:
            self.cols = np.array([0, self.nv], dtype=np.int64)
            self.send_sizes = self.recv_sizes = [int(lp[-1])]
            self.map = owner_map(self.nv, 0, self.nv, [counts], [rows])
            return
        total = counts.clone()
        dist.all_reduce(total, group=group)
        c = split_columns(total.cpu().numpy(), self.world)
        self.cols = c
        lo, hi = int(c[self.rank]), int(c[self.rank + 1])
        self.send_sizes = [int(lp[c[q + 1]] - lp[c[q]]) for q in range(self.world)]
        ncols = hi - lo
        cnt_in = torch.empty(self.world * ncols, dtype=torch.int64, device=device)
        dist.all_to_all_single(cnt_in, counts, [ncols] * self.world,
                               [int(c[q + 1] - c[q]) for q in range(self.world)], group=group)
        cnt_in = cnt_in.view(self.world, ncols)
        self.recv_sizes = [int(x) for x in cnt_in.sum(1).cpu()]
        rows_in = torch.empty(sum(self.recv_sizes), dtype=torch.int32, device=device)
        dist.all_to_all_single(rows_in, rows, self.recv_sizes, self.send_sizes, group=group)
        self.map = owner_map(self.nv, lo, hi, list(cnt_in), list(torch.split(rows_in, self.recv_sizes)))

    @property
    def col_range(self):
        return self.map.col_lo, self.map.col_hi

    def combine(self, partial):
        """This rank's owned values from every rank's partial values (local CSC order)."""
        import torch
        import torch.distributed as dist
        if self.single:
            return combine(self.map, [partial])
        vin = torch.empty(sum(self.recv_sizes), dtype=torch.float64, device=partial.device)
        dist.all_to_all_single(vin, partial, self.recv_sizes, self.send_sizes, group=self.group)
        return combine(self.map, list(torch.split(vin, self.recv_sizes)))

    def assemble(self, owned, dst: int = 0):
        """The whole CSC matrix (indptr int64, indices int32, values float64, numpy) on rank dst,
        None elsewhere; point-to-point sends of every owner's columns, for callers that want one
        matrix."""
        import torch
        import torch.distributed as dist
        if self.single:
            return self.map.indptr.cpu().numpy(), self.map.indices.cpu().numpy(), owned.cpu().numpy()
        dev = owned.device
        sizes = torch.zeros(self.world, dtype=torch.int64, device=dev)
        sizes[self.rank] = self.map.nnz
        dist.all_reduce(sizes, group=self.group)
        if self.rank != dst:
            to = _global(self.group, dst)
            dist.send(self.map.indptr.contiguous(), to, group=self.group)
            dist.send(self.map.indices.contiguous(), to, group=self.group)
            dist.send(owned.contiguous(), to, group=self.group)
            return None
        ptrs, rows, vals = [], [], []
        for q in range(self.world):
            ncols = int(self.cols[q + 1] - self.cols[q])
            if q == dst:
                p, r, v = self.map.indptr, self.map.indices, owned
            else:
                n = int(sizes[q])
                p = torch.empty(ncols + 1, dtype=torch.int64, device=dev)
                r = torch.empty(n, dtype=torch.int32, device=dev)
                v = torch.empty(n, dtype=torch.float64, device=dev)
                src = _global(self.group, q)
                dist.recv(p, src, group=self.group)
                dist.recv(r, src, group=self.group)
                dist.recv(v, src, group=self.group)
            ptrs.append(p.cpu().numpy())
            rows.append(r.cpu().numpy())
            vals.append(v.cpu().numpy())
        indptr = np.zeros(self.nv + 1, dtype=np.int64)
        base = 0
        for q in range(self.world):
            lo, hi = int(self.cols[q]), int(self.cols[q + 1])
            indptr[lo + 1:hi + 1] = base + ptrs[q][1:]
            base += int(ptrs[q][-1])
        return indptr, np.concatenate(rows), np.concatenate(vals)


class ShardedSearchlights:
    """Searchlight Procrustes of one hemisphere over the ranks of a torch.distributed group, one
    GPU per rank. Every rank holds the full X and Y on its GPU (nt x nv float64, column-major)
    and gets the CSC values of the columns it owns."""

    def __init__(self, nt, nv, indices, offsets, dists=None, radius=0.0, weights=None, group=None):
        import torch
        from .plan import Plan
        self.nt, self.nv = int(nt), int(nv)
        world, rank = _world_rank(group)
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        off = np.ascontiguousarray(offsets, dtype=np.int32)
        w = (hemisphere_weights(idx, off, dists, radius, nv) if weights is None
             else np.ascontiguousarray(weights, dtype=np.float64))
        self.bounds = split_searchlights(off, world)
        lo, hi = int(self.bounds[rank]), int(self.bounds[rank + 1])
        self.plan = None
        if hi > lo:
            sidx, soff, sw = sub_geometry(idx, off, w, lo, hi)
            self.plan = Plan(nt, nv, sidx, soff, weights=sw)
            indptr, rows = self.plan.pattern()
        else:
            indptr, rows = np.zeros(self.nv + 1, dtype=np.int64), np.zeros(0, dtype=np.int32)
        self.exchange = ColumnExchange(indptr, rows, nv, group, device="cuda")
        self.partial = torch.zeros(int(indptr[-1]), dtype=torch.float64, device="cuda")

    @property
    def col_range(self):
        return self.exchange.col_range

    def procrustes(self, d_X, d_Y, reflection=True, scaling=False, solver=L.SOLVER_MIXED):
        """Owned CSC values (float64, on this rank's GPU) of the hemisphere's Procrustes result."""
        import torch
        self.partial.zero_()
        if self.plan is not None:
            self.plan.procrustes_device(d_X.data_ptr(), d_Y.data_ptr(), self.partial.data_ptr(), reflection, scaling,
                                        solver, L.OUT_CSC, torch.cuda.current_stream().cuda_stream)
        return self.exchange.combine(self.partial)

    def close(self):
        if self.plan is not None:
            self.plan.close()
            self.plan = None
