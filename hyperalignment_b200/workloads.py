"""Seeded synthetic workloads for the searchlight alignment path.

The reference's public benchmark (StudyForrest surfaces loaded through
``neuroboros``, benchmark_neuroboros.py:99-153) is not available offline, so
these generators stand in for it with the same shapes: cortical vertices on a
Fibonacci-lattice unit sphere, one searchlight centred at every vertex, and
subject time series related by block-local orthogonal rotations.  No dataset
items are reproduced; everything is drawn from ``numpy.random.default_rng``.

Layouts follow the reference wrapper (hyperalignment_c.py:156-171): X, Y are
``nt x nv`` float64, searchlights are flattened to ``indices`` / ``offsets`` /
``dists`` int32/int32/float64 arrays, indices ascending within a searchlight.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
from scipy.spatial import cKDTree


@dataclasses.dataclass
class Searchlights:
    """Flat searchlight definition (the wrapper's layout, hyperalignment_c.py:161-171)."""

    indices: np.ndarray  # int32, concatenated vertex indices (sorted within each searchlight)
    offsets: np.ndarray  # int32, count + 1 entries, offsets[0] = 0
    dists: np.ndarray | None  # float64 geodesic distance to the centre, or None (uniform)
    radius: float
    nv: int

    @property
    def count(self) -> int:
        return int(self.offsets.size - 1)

    @property
    def sizes(self) -> np.ndarray:
        return np.diff(self.offsets).astype(np.int32)

    def as_lists(self):
        sls = [self.indices[self.offsets[s]:self.offsets[s + 1]] for s in range(self.count)]
        if self.dists is None:
            return sls, None
        ds = [self.dists[self.offsets[s]:self.offsets[s + 1]] for s in range(self.count)]
        return sls, ds

    def subset(self, which: np.ndarray) -> "Searchlights":
        """Searchlights ``which`` (in that order), same vertex space."""
        which = np.asarray(which, dtype=np.int64)
        sizes = self.sizes[which]
        offs = np.zeros(which.size + 1, dtype=np.int32)
        np.cumsum(sizes, out=offs[1:])
        idx = np.concatenate([self.indices[self.offsets[s]:self.offsets[s + 1]] for s in which])
        d = None
        if self.dists is not None:
            d = np.concatenate([self.dists[self.offsets[s]:self.offsets[s + 1]] for s in which])
        return Searchlights(idx.astype(np.int32), offs, d, self.radius, self.nv)


def fibonacci_sphere(n: int) -> np.ndarray:
    """``n`` points on the unit sphere: phi = arccos(1 - 2(i+1/2)/n), theta = pi(1+sqrt5)(i+1/2)."""
    i = np.arange(n, dtype=np.float64) + 0.5
    phi = np.arccos(1.0 - 2.0 * i / n)
    theta = math.pi * (1.0 + math.sqrt(5.0)) * i
    return np.stack([np.cos(theta) * np.sin(phi), np.sin(theta) * np.sin(phi), np.cos(phi)], axis=1)


def _geodesic(chord: np.ndarray) -> np.ndarray:
    return 2.0 * np.arcsin(np.clip(chord * 0.5, 0.0, 1.0))


def _pack(rows, dists_rows, nv: int) -> Searchlights:
    order = [np.argsort(r, kind="stable") for r in rows]
    rows = [np.asarray(r)[o] for r, o in zip(rows, order)]
    dists_rows = [np.asarray(d)[o] for d, o in zip(dists_rows, order)]
    sizes = np.array([len(r) for r in rows], dtype=np.int64)
    offs = np.zeros(len(rows) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offs[1:])
    if offs[-1] >= 2**31:
        raise ValueError("searchlight index total exceeds int32")
    idx = np.concatenate(rows).astype(np.int32)
    d = np.concatenate(dists_rows).astype(np.float64)
    radius = 1.0001 * float(d.max())
    return Searchlights(idx, offs.astype(np.int32), d, radius, nv)


def searchlights_disc(points: np.ndarray, radius: float) -> Searchlights:
    """Geodesic disc of ``radius`` radians around every vertex."""
    tree = cKDTree(points)
    chord = 2.0 * math.sin(radius / 2.0)
    rows = tree.query_ball_point(points, r=chord)
    dists = []
    for c, r in enumerate(rows):
        r = np.asarray(r, dtype=np.int64)
        dists.append(_geodesic(np.linalg.norm(points[r] - points[c], axis=1)))
    return _pack(rows, dists, points.shape[0])


def searchlights_knn(points: np.ndarray, sizes: np.ndarray) -> Searchlights:
    """k-nearest-neighbour searchlight of ``sizes[c]`` vertices around every vertex ``c``."""
    tree = cKDTree(points)
    kmax = int(sizes.max())
    chord, nn = tree.query(points, k=kmax)
    rows, dists = [], []
    for c in range(points.shape[0]):
        k = int(sizes[c])
        rows.append(nn[c, :k])
        dists.append(_geodesic(chord[c, :k]))
    return _pack(rows, dists, points.shape[0])


@dataclasses.dataclass
class BlockRotation:
    """Block-diagonal orthogonal map in vertex space: Voronoi cells of a coarse lattice."""

    cells: list  # list of int64 vertex-index arrays
    mats: list  # list of (k, k) orthogonal matrices

    def apply(self, X: np.ndarray) -> np.ndarray:
        Y = np.empty_like(X)
        for cell, Q in zip(self.cells, self.mats):
            Y[:, cell] = X[:, cell] @ Q
        return Y


def block_rotation(points: np.ndarray, rng: np.random.Generator, verts_per_cell: int = 64) -> BlockRotation:
    nv = points.shape[0]
    seeds = fibonacci_sphere(max(1, nv // verts_per_cell))
    _, owner = cKDTree(seeds).query(points, k=1)
    cells, mats = [], []
    for c in range(seeds.shape[0]):
        cell = np.flatnonzero(owner == c)
        if cell.size == 0:
            continue
        g = rng.standard_normal((cell.size, cell.size))
        q, r = np.linalg.qr(g)
        q = q * np.sign(np.diag(r))[np.newaxis, :]
        cells.append(cell)
        mats.append(q)
    return BlockRotation(cells, mats)


def zscore_columns(X: np.ndarray) -> np.ndarray:
    """Population z-score of each column (ha_linalg.c:263-291 semantics, var < 1e-30 -> 0)."""
    m = X.mean(axis=0)
    v = (X * X).mean(axis=0) - m * m
    inv = np.where(v < 1e-30, 0.0, 1.0 / np.sqrt(np.maximum(v, 1e-300)))
    return (X - m) * inv


@dataclasses.dataclass
class Workload:
    name: str
    X: np.ndarray  # nt x nv float64 (C order)
    Y: np.ndarray  # nt x nv float64
    sls: Searchlights
    reflection: bool
    scaling: bool
    extra: dict = dataclasses.field(default_factory=dict)

    @property
    def nt(self) -> int:
        return int(self.X.shape[0])

    @property
    def nv(self) -> int:
        return int(self.X.shape[1])


def plain_procrustes(seed: int = 0, nv: int = 2562, nt: int = 200, radius: float = 0.343) -> Workload:
    """Plain searchlight Procrustes: X ~ N(0,1) z-scored, Y = X R + 0.1 N(0,1).

    nv = 2562, nt = 200 and a 0.343 rad geodesic disc give searchlights of
    71-78 vertices; reflection allowed, no scaling.
    """
    rng = np.random.default_rng(seed)
    pts = fibonacci_sphere(nv)
    sls = searchlights_disc(pts, radius)
    X = zscore_columns(rng.standard_normal((nt, nv)))
    R = block_rotation(pts, rng)
    Y = R.apply(X) + 0.1 * rng.standard_normal((nt, nv))
    return Workload("plain_procrustes", np.ascontiguousarray(X), np.ascontiguousarray(Y), sls, True, False)


def _uniform_sizes(rng, nv, lo, hi):
    return rng.integers(lo, hi + 1, size=nv)


def hemisphere_subjects(seed: int = 0, nv: int = 10242, nt: int = 400, n_subj: int = 10,
                        size_lo: int = 100, size_hi: int = 300, noise: float = 0.2,
                        ar_rho: float = 0.0, noise_span: float = 1.0):
    """Shared N(0,1) latent time series times per-subject block-local rotations plus noise.

    Returns (points, searchlights, list of subject matrices nt x nv).  With
    ``ar_rho`` > 0 the noise is AR(1): e_t = rho e_{t-1} + sqrt(1 - rho^2) eps_t.  With
    ``noise_span`` > 1 the noise amplitude varies smoothly over the sphere, from ``noise`` at
    the south pole to ``noise * noise_span`` at the north pole (log-linear in z).
    """
    rng = np.random.default_rng(seed)
    pts = fibonacci_sphere(nv)
    sls = searchlights_knn(pts, _uniform_sizes(rng, nv, size_lo, size_hi))
    L = rng.standard_normal((nt, nv))
    subjects = []
    for _ in range(n_subj):
        R = block_rotation(pts, rng)
        eps = rng.standard_normal((nt, nv))
        if ar_rho > 0.0:
            e = np.empty_like(eps)
            e[0] = eps[0]
            c = math.sqrt(1.0 - ar_rho * ar_rho)
            for t in range(1, nt):
                e[t] = ar_rho * e[t - 1] + c * eps[t]
            eps = e
        amp = noise * noise_span ** ((pts[:, 2] + 1.0) / 2.0) if noise_span != 1.0 else noise
        subjects.append(np.ascontiguousarray(R.apply(L) + amp * eps))
    return pts, sls, subjects


def template_procrustes_pair(seed: int = 0, nv: int = 10242, nt: int = 400) -> Workload:
    """One searchlight solve of the hemisphere template loop: subject 1 onto subject 0, with scaling."""
    _, sls, subj = hemisphere_subjects(seed, nv=nv, nt=nt, n_subj=2)
    return Workload("template_procrustes", subj[1], subj[0], sls, True, True)


GRID_ALPHAS = np.logspace(-3.0, 3.0, 10)   # 10 log-spaced ridge penalties in [1e-3, 1e3]
GRID_NPCS = np.array([10, 20, 50, 1 << 30], dtype=np.int32)  # PC counts; the last is "all" (clipped at K)


def ridge_grid_pair(seed: int = 0, nv: int = 40962, nt: int = 500, size_lo: int = 50, size_hi: int = 500,
                    n_subj: int = 2, pair=(0, 1), noise: float = 0.2, noise_span: float = 1.0) -> Workload:
    """Searchlight ridge grid search inputs: subjects of the hemisphere generator with AR(1)
    noise (rho 0.5), searchlight sizes uniform in [size_lo, size_hi]; X = subject pair[0],
    Y = subject pair[1] (the ridge predicts Y's searchlight columns from X's)."""
    _, sls, subj = hemisphere_subjects(seed, nv=nv, nt=nt, n_subj=n_subj, size_lo=size_lo, size_hi=size_hi,
                                       ar_rho=0.5, noise=noise, noise_span=noise_span)
    return Workload("ridge_grid", subj[pair[0]], subj[pair[1]], sls, True, False)


def duplicate_columns(X: np.ndarray, sls: Searchlights, frac: float, rng) -> np.ndarray:
    """Copy one member's column onto another in about ``frac * count / 4`` random searchlights.

    Every searchlight that holds both vertices of a copied pair becomes exactly rank-deficient;
    with overlapping searchlights that is usually far more than ``frac`` of them (see
    duplicate_columns_to_fraction for a set fraction).  Returns the mask of those searchlights.
    """
    nv = X.shape[1]
    dup_of = -np.ones(nv, dtype=np.int64)
    chosen = rng.choice(sls.count, size=max(1, int(frac * sls.count / 4)), replace=False)
    for s in chosen:
        sl = sls.indices[sls.offsets[s]:sls.offsets[s + 1]]
        a, b = rng.choice(sl.size, size=2, replace=False)
        v1, v2 = int(sl[a]), int(sl[b])
        if dup_of[v1] >= 0 or dup_of[v2] >= 0 or (dup_of == v2).any():
            continue
        X[:, v2] = X[:, v1]
        dup_of[v2] = v1
    mask = np.zeros(sls.count, dtype=bool)
    dups = np.flatnonzero(dup_of >= 0)
    for s in range(sls.count):
        sl = sls.indices[sls.offsets[s]:sls.offsets[s + 1]]
        inside = np.isin(dups, sl)
        if inside.any():
            mask[s] = np.isin(dup_of[dups[inside]], sl).any()
    return mask


def duplicate_columns_to_fraction(X: np.ndarray, sls: Searchlights, frac: float, rng) -> np.ndarray:
    """Copy columns pair by pair until about ``frac`` of the searchlights are rank-deficient.

    Each step picks a not yet singular searchlight and two of its members that are in no earlier
    pair, copies one column onto the other, and marks every searchlight holding both.  Returns
    the exact mask of singular searchlights.
    """
    nv = X.shape[1]
    order = np.argsort(sls.indices, kind="stable")
    owner = np.repeat(np.arange(sls.count), np.diff(sls.offsets))[order]
    starts = np.searchsorted(sls.indices[order], np.arange(nv + 1))
    members = [owner[starts[v]:starts[v + 1]] for v in range(nv)]  # searchlights holding v
    mask = np.zeros(sls.count, dtype=bool)
    used = np.zeros(nv, dtype=bool)
    target = frac * sls.count
    for _ in range(20 * sls.count):
        if mask.sum() >= target:
            break
        s = int(rng.integers(sls.count))
        if mask[s]:
            continue
        sl = sls.indices[sls.offsets[s]:sls.offsets[s + 1]]
        a, b = rng.choice(sl.size, size=2, replace=False)
        v1, v2 = int(sl[a]), int(sl[b])
        if used[v1] or used[v2]:
            continue
        X[:, v2] = X[:, v1]
        used[v1] = used[v2] = True
        mask[np.intersect1d(members[v1], members[v2])] = True
    return mask


def rank_deficient_pair(seed: int = 0, nv: int = 10242, nt: int = 400, frac: float = 0.10) -> Workload:
    """Template pair with duplicated vertex columns so about ``frac`` of searchlights are singular."""
    w = template_procrustes_pair(seed, nv=nv, nt=nt)
    rng = np.random.default_rng(seed + 1000)
    X = w.X.copy()
    mask = duplicate_columns_to_fraction(X, w.sls, frac, rng)
    return Workload("rank_deficient", X, w.Y, w.sls, True, True, {"singular": mask})


def forrest_shaped(seed: int = 0, nv: int = 9675, nt: int = 1818) -> Workload:
    """Shapes of the reference's published StudyForrest run: nt = 1818, about 9,675 searchlights of ~121 (90-170)."""
    rng = np.random.default_rng(seed)
    pts = fibonacci_sphere(nv)
    sls = searchlights_knn(pts, _uniform_sizes(rng, nv, 90, 170))
    X = zscore_columns(rng.standard_normal((nt, nv)))
    R = block_rotation(pts, rng)
    Y = R.apply(X) + 0.1 * rng.standard_normal((nt, nv))
    return Workload("forrest_shaped", X, Y, sls, True, False)


def small_case(seed: int = 0, nv: int = 162, nt: int = 40, lo: int = 8, hi: int = 24,
               reflection: bool = True, scaling: bool = False) -> Workload:
    """Small k-NN case for parity tests (seconds on the CPU oracle)."""
    rng = np.random.default_rng(seed)
    pts = fibonacci_sphere(nv)
    sls = searchlights_knn(pts, _uniform_sizes(rng, nv, lo, hi))
    X = zscore_columns(rng.standard_normal((nt, nv)))
    R = block_rotation(pts, rng, verts_per_cell=16)
    Y = R.apply(X) + 0.1 * rng.standard_normal((nt, nv))
    return Workload("small", np.ascontiguousarray(X), np.ascontiguousarray(Y), sls, reflection, scaling)
