"""CPU oracle: a numpy restatement of the reference's searchlight alignment path.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, always as the checker; the product path (the CUDA
library) never calls it.

Every function follows the reference C library (neurolabusc/hyperalignment,
csrc/) in float64 and cites the lines it restates.  Pinning: tests/test_oracle.py
checks these functions against the reference's own known-answer tests
(csrc/ha_test.c) and against golden vectors produced by the compiled reference
(tests/golden/make_golden.py, oracle/Makefile).  The SVD is LAPACK gesdd through
numpy (the reference calls dgesdd_ / dgesvd_, csrc/ha_linalg.c:53-89).
"""

from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------------------------------------
# deterministic test RNG of the reference harness (csrc/ha_test.c:33-65)
# ---------------------------------------------------------------------------------------------

class SplitMix64:
    """splitmix64 stream with the harness's uniform and Box-Muller normal draws."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.state = seed & self.MASK

    def next(self) -> int:  # csrc/ha_test.c:41-47
        self.state = (self.state + 0x9E3779B97F4A7C15) & self.MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:  # csrc/ha_test.c:50-52
        return (self.next() >> 11) / float(1 << 53)

    def randn(self) -> float:  # csrc/ha_test.c:55-60
        u1 = self.uniform()
        u2 = self.uniform()
        if u1 < 1e-15:
            u1 = 1e-15
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)

    def fill(self, rows: int, cols: int) -> np.ndarray:  # csrc/ha_test.c:63-66 (row-major fill)
        return np.array([self.randn() for _ in range(rows * cols)], dtype=np.float64).reshape(rows, cols)


# ---------------------------------------------------------------------------------------------
# weights (csrc/ha_searchlight.c:970-1001, :36-92)
# ---------------------------------------------------------------------------------------------

def searchlight_weights(idx: np.ndarray, off: np.ndarray, dists, radius: float, nv: int) -> np.ndarray:
    """Flat weights, same operation order as the reference (vertex sums in flat order)."""
    idx = np.asarray(idx, dtype=np.int64)
    vsum = np.zeros(nv, dtype=np.float64)
    if dists is None:
        w = np.ones(idx.size, dtype=np.float64)
    else:
        w = (radius - np.asarray(dists, dtype=np.float64)) / radius
    np.add.at(vsum, idx, w)  # sequential, in flat order, like the C loop
    return w / vsum[idx]


# ---------------------------------------------------------------------------------------------
# local Procrustes (csrc/ha_procrustes.c:17-127; column-major twin csrc/ha_searchlight.c:578-659)
# ---------------------------------------------------------------------------------------------

def _det_sign_lu(T: np.ndarray) -> float:
    """Sign of det(T) from LU with partial pivoting (the dgetrf_ test of csrc/ha_procrustes.c:56-79)."""
    sign, _ = np.linalg.slogdet(T)
    return float(sign)


def procrustes(X: np.ndarray, Y: np.ndarray, reflection: bool = True, scaling: bool = False,
               return_svd: bool = False):
    """T = U V^T for X^T Y = U S V^T, with the reference's reflection and scaling rules."""
    A = X.T @ Y
    U, s, Vt = np.linalg.svd(A)
    T = U @ Vt
    s = s.copy()
    if not reflection:
        if _det_sign_lu(T) < 0:  # csrc/ha_procrustes.c:80-94
            s[-1] *= -1.0
            T = T - 2.0 * np.outer(U[:, -1], Vt[-1, :])
    if scaling:  # csrc/ha_procrustes.c:98-120: population variance of the local X columns
        var_sum = float(np.sum(np.var(X, axis=0)))
        T = T * (s.sum() / (var_sum * X.shape[0]))
    if return_svd:
        return T, U, s, Vt
    return T


def local_transforms(X, Y, idx, off, reflection=True, scaling=False):
    """Per-searchlight local transforms T_s (n_s x n_s), unweighted."""
    out = []
    for s in range(len(off) - 1):
        sl = idx[off[s]:off[s + 1]]
        out.append(procrustes(X[:, sl], Y[:, sl], reflection, scaling))
    return out


def searchlight_procrustes_dense(X, Y, idx, off, dists, radius, reflection=True, scaling=False,
                                 T_out=None, transforms=None):
    """Dense searchlight Procrustes, csrc/ha_searchlight.c:950-1100 (cpu64 arm).

    T_out[sl[i], sl[j]] += w[i] * T_s[i, j] with row weights (csrc/ha_searchlight.c:1073-1085).
    """
    nt, nv = X.shape
    w = searchlight_weights(idx, off, dists, radius, nv)
    if T_out is None:
        T_out = np.zeros((nv, nv), dtype=np.float64)
    for s in range(len(off) - 1):
        sl = idx[off[s]:off[s + 1]]
        T = transforms[s] if transforms is not None else procrustes(X[:, sl], Y[:, sl], reflection, scaling)
        T_out[np.ix_(sl, sl)] += T * w[off[s]:off[s + 1], np.newaxis]
    return T_out


# ---------------------------------------------------------------------------------------------
# CSC pattern and scatter (csrc/ha_sparse.c)
# ---------------------------------------------------------------------------------------------

def sparse_init(idx, off, nv):
    """CSC pattern of the union of sl x sl blocks: (col, row)-sorted unique pairs, csrc/ha_sparse.c:31-112."""
    keys = []
    for s in range(len(off) - 1):
        sl = np.asarray(idx[off[s]:off[s + 1]], dtype=np.int64)
        rows = np.repeat(sl, sl.size)
        cols = np.tile(sl, sl.size)
        keys.append(cols * nv + rows)
    keys = np.unique(np.concatenate(keys))
    cols = keys // nv
    rows = (keys - cols * nv).astype(np.int32)
    indptr = np.zeros(nv + 1, dtype=np.int64)
    np.add.at(indptr, cols + 1, 1)
    indptr = np.cumsum(indptr)
    return indptr.astype(np.int32), rows


def sparse_scatter_add(indptr, indices, data, sl_rows, sl_cols, T, w=None):
    """data[(sl_rows[i], sl_cols[j])] += T[i, j] * w[i], skipping absent entries (csrc/ha_sparse.c:128-142)."""
    for j, col in enumerate(sl_cols):
        a, b = int(indptr[col]), int(indptr[col + 1])
        rows = indices[a:b]
        pos = np.searchsorted(rows, sl_rows)
        ok = (pos < rows.size)
        ok[ok] = rows[pos[ok]] == np.asarray(sl_rows)[ok]
        vals = T[:, j] * (w if w is not None else 1.0)
        np.add.at(data, a + pos[ok], vals[ok])
    return data


def searchlight_procrustes_csc(X, Y, idx, off, indptr, indices, data, weights=None, reflection=True,
                               scaling=False, transforms=None):
    """Sparse-API searchlight Procrustes, csrc/ha_searchlight.c:147-201 (cpu64 arm), sls_Y = sls_X."""
    for s in range(len(off) - 1):
        sl = idx[off[s]:off[s + 1]]
        T = transforms[s] if transforms is not None else procrustes(X[:, sl], Y[:, sl], reflection, scaling)
        w = None if weights is None else weights[off[s]:off[s + 1]]
        sparse_scatter_add(indptr, indices, data, sl, sl, T, w)
    return data


# ---------------------------------------------------------------------------------------------
# ridge (csrc/ha_ridge.c:13-54) and searchlight ridge (csrc/ha_searchlight.c:1378-1429)
# ---------------------------------------------------------------------------------------------

def ridge(X, Y, alpha):
    """betas = V diag(s / (alpha + s^2)) U^T Y with the thin SVD X = U diag(s) V^T."""
    U, s, Vt = np.linalg.svd(X, full_matrices=False)
    d = s / (alpha + s * s)
    return Vt.T @ (d[:, np.newaxis] * (U.T @ Y))


def searchlight_ridge_csc(X, Y, idx, off, indptr, indices, data, alpha, weights=None):
    for s in range(len(off) - 1):
        sl = idx[off[s]:off[s + 1]]
        T = ridge(X[:, sl], Y[:, sl], alpha)
        w = None if weights is None else weights[off[s]:off[s + 1]]
        sparse_scatter_add(indptr, indices, data, sl, sl, T, w)
    return data


# ---------------------------------------------------------------------------------------------
# ridge grid (csrc/ha_ridge.c:97-227), ensemble ridge (csrc/ha_ridge.c:229-345), CV split indices
# (csrc/ha_ensemble.c:12-249), and their composition over searchlights
# ---------------------------------------------------------------------------------------------

def ridge_grid(X, y, alphas, npcs, train_idx=None):
    """betas[v, a, p] (a trailing target axis when y is 2-D), csrc/ha_ridge.c:97-227.

    Thin SVD of the training rows; d[k, a] = s_k / (alpha_a + s_k^2) times U^T y; the PC chunk
    [npcs[p-1], npcs[p]) clipped at K = min(rows, cols) is summed into slot p (empty chunks leave
    it zero), then the slots are summed cumulatively over p.
    """
    alphas = np.asarray(alphas, dtype=np.float64)
    Xt = X if train_idx is None else X[np.asarray(train_idx)]
    yt = y if train_idx is None else y[np.asarray(train_idx)]
    U, s, Vt = np.linalg.svd(Xt, full_matrices=False)
    K = s.size
    d = s[:, None] / (alphas[None, :] + (s * s)[:, None])  # K x A
    uty = U.T @ yt                                           # K (x T)
    dut = d * uty[:, None] if uty.ndim == 1 else d[:, :, None] * uty[:, None, :]
    N = X.shape[1]
    betas = np.zeros((N, alphas.size, len(npcs)) + uty.shape[1:])
    prev = 0
    for p, cur in enumerate(npcs):
        cur = int(cur)
        if cur - prev > 0 and prev < K:
            end = min(cur, K)
            betas[:, :, p] = np.tensordot(Vt[prev:end].T, dut[prev:end], axes=(1, 0))
        prev = cur
    return np.cumsum(betas, axis=2)


def ensemble_ridge(X, y, alphas, npcs, train_li, test_li):
    """csrc/ha_ridge.c:229-345 with y of one target (1-D) or several (2-D, cost summed over them).

    Returns (weights, pred, r2, alpha, npc, best, cost): the model-averaged betas of the winner,
    its averaged test predictions, 1 - cost / sum(y^2), and the full cost grid (A x P).
    """
    alphas = np.asarray(alphas, dtype=np.float64)
    nt = X.shape[0]
    A, P = alphas.size, len(npcs)
    tshape = y.shape[1:]
    wsum = None
    psum = np.zeros((nt, A, P) + tshape)
    count = np.zeros(nt, dtype=np.int64)
    for tr, te in zip(train_li, test_li):
        b = ridge_grid(X, y, alphas, npcs, tr)
        wsum = b.copy() if wsum is None else wsum + b
        te = np.asarray(te, dtype=np.int64)
        if te.size:
            # pred[t, a, p(, target)] = sum_v X[t, v] b[v, a, p(, target)]  (csrc/ha_ridge.c:297-303)
            psum[te] += (X[te] @ b.reshape(b.shape[0], -1)).reshape((te.size,) + b.shape[1:])
            count[te] += 1
    weights_avg = wsum / len(train_li)
    pred = np.zeros_like(psum)
    hit = count > 0
    pred[hit] = psum[hit] / count[hit].reshape((-1,) + (1,) * (psum.ndim - 1))
    diff = y.reshape((nt, 1, 1) + tshape) - pred
    cost = (diff * diff).reshape(nt, A, P, -1).sum(axis=(0, 3))
    best = int(np.argmin(cost.ravel()))  # first minimum, csrc/ha_ridge.c:322-327
    ba, bp = divmod(best, P)
    r2 = 1.0 - cost.ravel()[best] / float((y * y).sum())
    return weights_avg[:, ba, bp], pred[:, ba, bp], r2, float(alphas[ba]), int(npcs[bp]), best, cost


def searchlight_ridge_grid_csc(X, Y, idx, off, indptr, indices, data, alphas, npcs, train_li, test_li,
                               weights=None):
    """Per searchlight: ensemble_ridge of X[:, sl] on the n targets Y[:, sl] (one winner per
    searchlight, cost summed over the targets), the winner's betas scattered like the ridge solve
    (csrc/ha_searchlight.c:1378-1429).  Returns (data, best[count], cost[count, A, P])."""
    count = len(off) - 1
    best = np.zeros(count, dtype=np.int32)
    costs = np.zeros((count, len(alphas), len(npcs)))
    for s in range(count):
        sl = idx[off[s]:off[s + 1]]
        B, _, _, _, _, b, c = ensemble_ridge(X[:, sl], Y[:, sl], alphas, npcs, train_li, test_li)
        best[s] = b
        costs[s] = c
        w = None if weights is None else weights[off[s]:off[s + 1]]
        sparse_scatter_add(indptr, indices, data, sl, sl, B, w)
    return data, best, costs


def ridge_features(X, idx, off, rows, n_sv=64):
    """Perceptron features per searchlight: the n_sv largest singular values of X[rows, sl]
    divided by the largest (zero-padded), then log n."""
    out = np.zeros((len(off) - 1, n_sv + 1))
    Xr = X[np.asarray(rows)]
    for s in range(len(off) - 1):
        sl = idx[off[s]:off[s + 1]]
        sv = np.linalg.svd(Xr[:, sl], compute_uv=False)
        k = min(n_sv, sv.size)
        if sv[0] > 0:
            out[s, :k] = sv[:k] / sv[0]
        out[s, n_sv] = math.log(sl.size)
    return out


def searchlight_ridge_at(X, Y, idx, off, indptr, indices, data, alphas, npcs, rows, choice, weights=None):
    """ha_ridge_grid's beta at grid point choice[s] (g = a * len(npcs) + p), fitted on the rows,
    of every searchlight's targets, scattered like the ridge solve."""
    P = len(npcs)
    for s in range(len(off) - 1):
        sl = idx[off[s]:off[s + 1]]
        a, p = divmod(int(choice[s]), P)
        B = ridge_grid(X[:, sl], Y[:, sl], alphas, npcs, rows)[:, a, p, :]
        w = None if weights is None else weights[off[s]:off[s + 1]]
        sparse_scatter_add(indptr, indices, data, sl, sl, B, w)
    return data


class Xoshiro256:
    """xoshiro256** seeded by splitmix64, modulo range reduction (csrc/ha_ensemble.c:12-46)."""
    M = (1 << 64) - 1

    def __init__(self, seed: int):
        self.s = []
        seed &= self.M
        for _ in range(4):
            seed = (seed + 0x9E3779B97F4A7C15) & self.M
            z = seed
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
            self.s.append(z ^ (z >> 31))

    @staticmethod
    def _rotl(x, k):
        return ((x << k) | (x >> (64 - k))) & Xoshiro256.M

    def next(self) -> int:
        s = self.s
        out = (self._rotl((s[1] * 5) & self.M, 7) * 9) & self.M
        t = (s[1] << 17) & self.M
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = self._rotl(s[3], 45)
        return out

    def below(self, n: int) -> int:
        return self.next() % n


def ensemble_indices(nt, n_perms, n_folds, blocksize, buffersize, seed, mask=None):
    """CV splits of csrc/ha_ensemble.c:58-249, draw for draw.  Returns (train_li, test_li)."""
    rng = Xoshiro256(seed)
    n_blocks, remainder = nt // blocksize, nt % blocksize
    padded = nt + 2 * buffersize
    mapping = None
    if mask is not None:
        mask = np.asarray(mask, dtype=bool)
        mapping = np.full(nt, -1, dtype=np.int64)
        mapping[mask] = np.arange(int(mask.sum()))
    train_li, test_li = [], []

    def block_out(mk, centre):
        lo = max(centre, 0)
        hi = min(centre + 2 * buffersize, padded - 1)
        mk[lo:hi + 1] = False

    for _ in range(n_perms):
        shift = rng.below(remainder + 1)
        order = list(range(n_blocks))
        for i in range(n_blocks - 1, 0, -1):
            j = rng.below(i + 1)
            order[i], order[j] = order[j], order[i]
        f0 = 0
        for fold in range(n_folds):
            f1 = (fold + 1) * n_blocks // n_folds
            test_raw = [order[b] * blocksize + k + shift for b in range(f0, f1) for k in range(blocksize)]
            test_raw = [t for t in test_raw if t < nt]
            trm = np.ones(padded, dtype=bool)
            for t in test_raw:
                block_out(trm, t)
            if mask is not None:
                trm[buffersize:buffersize + nt][~mask] = False
            valid = np.flatnonzero(trm[buffersize:buffersize + nt])
            if valid.size == 0:
                raise ValueError("fold without training rows")
            train = np.array([valid[rng.below(valid.size)] for _ in range(nt)], dtype=np.int64)
            tem = np.ones(padded, dtype=bool)
            for i in np.flatnonzero(np.bincount(train, minlength=nt)):
                block_out(tem, int(i))
            if mask is not None:
                tem[buffersize:buffersize + nt][~mask] = False
            test = np.flatnonzero(tem[buffersize:buffersize + nt])
            if mapping is not None:
                train, test = mapping[train], mapping[test]
            train_li.append(train.astype(np.int32))
            test_li.append(test.astype(np.int32))
            f0 = f1
    return train_li, test_li


# ---------------------------------------------------------------------------------------------
# learned (alpha, PC count) proposal: the perceptron in float64 (no reference counterpart; the
# checker for the GPU forward / backward / inference kernels)
# ---------------------------------------------------------------------------------------------

MLP_IN, MLP_HIDDEN = 65, 128


def mlp_layout(C):
    """Offsets of W1[65][128], b1, W2[128][128], b2, W3[128][C], b3 in the packed parameters."""
    sizes = [("W1", MLP_IN * MLP_HIDDEN), ("b1", MLP_HIDDEN), ("W2", MLP_HIDDEN * MLP_HIDDEN), ("b2", MLP_HIDDEN),
             ("W3", MLP_HIDDEN * C), ("b3", C)]
    out, o = {}, 0
    for k, n in sizes:
        out[k] = (o, n)
        o += n
    out["total"] = o
    return out


def _unpack(params, C):
    L = mlp_layout(C)
    g = {k: np.asarray(params[L[k][0]:L[k][0] + L[k][1]], dtype=np.float64) for k in L if k != "total"}
    g["W1"] = g["W1"].reshape(MLP_IN, MLP_HIDDEN)
    g["W2"] = g["W2"].reshape(MLP_HIDDEN, MLP_HIDDEN)
    g["W3"] = g["W3"].reshape(MLP_HIDDEN, C)
    return g


def _gelu(z):
    from scipy.special import erf
    return 0.5 * z * (1.0 + erf(z / math.sqrt(2.0)))


def _gelu_grad(z):
    from scipy.special import erf
    return 0.5 * (1.0 + erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def mlp_forward(params, C, X):
    """Logits of x -> 128 GELU -> 128 GELU -> C for the rows of X (n x 65)."""
    g = _unpack(params, C)
    z1 = X @ g["W1"] + g["b1"]
    h1 = _gelu(z1)
    z2 = h1 @ g["W2"] + g["b2"]
    h2 = _gelu(z2)
    return h2 @ g["W3"] + g["b3"]


def mlp_loss_grad(params, C, X, y):
    """Mean softmax cross-entropy over the rows of X with labels y, and its gradient (packed)."""
    g = _unpack(params, C)
    n = X.shape[0]
    z1 = X @ g["W1"] + g["b1"]
    h1 = _gelu(z1)
    z2 = h1 @ g["W2"] + g["b2"]
    h2 = _gelu(z2)
    z3 = h2 @ g["W3"] + g["b3"]
    m = z3.max(axis=1, keepdims=True)
    lse = m[:, 0] + np.log(np.exp(z3 - m).sum(axis=1))
    loss = float(np.mean(lse - z3[np.arange(n), y]))
    d3 = np.exp(z3 - lse[:, None])
    d3[np.arange(n), y] -= 1.0
    d3 /= n
    dz2 = (d3 @ g["W3"].T) * _gelu_grad(z2)
    dz1 = (dz2 @ g["W2"].T) * _gelu_grad(z1)
    grads = {"W1": X.T @ dz1, "b1": dz1.sum(0), "W2": h1.T @ dz2, "b2": dz2.sum(0), "W3": h2.T @ d3, "b3": d3.sum(0)}
    L = mlp_layout(C)
    out = np.zeros(L["total"])
    for k in grads:
        o, cnt = L[k]
        out[o:o + cnt] = grads[k].ravel()
    return loss, out


# ---------------------------------------------------------------------------------------------
# z-score (csrc/ha_linalg.c:263-291)
# ---------------------------------------------------------------------------------------------

def aligned_correlation(X, Y, W=None):
    """Vertex-wise correlation of A = X @ W (A = X when W is None) with Y, the evaluation of
    benchmark_neuroboros.py:204-211 (np.mean(zscore(A, axis=0) * zscore(Y, axis=0), axis=0), scipy's
    population z-score; benchmark_neuroboros.py:229-232 forms X @ W). W: dense or scipy sparse."""
    import warnings
    from scipy.stats import zscore
    A = X if W is None else np.asarray(X @ W)
    with warnings.catch_warnings(), np.errstate(invalid="ignore", divide="ignore"):
        warnings.simplefilter("ignore", RuntimeWarning)  # a constant column: 0 / 0, NaN as in the reference
        return np.mean(zscore(A, axis=0) * zscore(Y, axis=0), axis=0)


def searchlight_pca_template(dms, idx, off, dists, radius):
    """Searchlight PCA template, src/hyperalignment/searchlight.py:215-236 with
    compute_template(kind="pca", max_npc=n, common_topography=True, demean=False)
    (src/hyperalignment/local_template.py:224-248, :72-78, :11-53).

    Per searchlight: X = [dms_1[:, sl], ..., dms_ns[:, sl]] (nt x ns*n); the local template is
    U_k S_k / sqrt(ns) for the top k = min(n, nt, ns*n) singular pairs of X; it is rotated by the
    Procrustes of the stacked template onto the stacked subjects, whose cross product is
    tmpl^T sum_s dms_s[:, sl] (src/hyperalignment/procrustes.py, reflection allowed, no scaling);
    the rotated template is added into the columns sl with the searchlight weights.

    The reference takes the top singular pairs from scikit-learn's randomized_svd (Halko,
    Martinsson and Tropp 2011; random_state=0, 4 or 7 power iterations, 10 oversamples). This
    restatement takes them from an exact SVD: the two agree where the top-k singular subspace is
    separated from the rest (pinned on such inputs); without a gap the reference's result depends
    on its random draws.
    """
    ns = len(dms)
    nt, nv = dms[0].shape
    w = searchlight_weights(idx, off, dists, radius, nv)
    tpl = np.zeros((nt, nv))
    for s in range(len(off) - 1):
        sl = np.asarray(idx[off[s]:off[s + 1]])
        X = np.hstack([d[:, sl] for d in dms])
        k = min(sl.size, nt, X.shape[1])
        U, sv, _ = np.linalg.svd(X, full_matrices=False)
        tmpl = U[:, :k] * (sv[:k] / np.sqrt(ns))
        M = np.sum([d[:, sl] for d in dms], axis=0)
        Ua, _, Vta = np.linalg.svd(tmpl.T @ M, full_matrices=False)
        tpl[:, sl] += (tmpl @ (Ua @ Vta)) * w[off[s]:off[s + 1]][np.newaxis]
    return tpl


def zscore_columns(X):
    """One-pass population z-score, var < 1e-30 -> 0 (csrc/ha_linalg.c:263-291)."""
    M = X.shape[0]
    sums = X.sum(axis=0)
    sum2 = (X * X).sum(axis=0)
    mean = sums * (1.0 / M)
    var = sum2 * (1.0 / M) - mean * mean
    inv = np.where(var < 1e-30, 0.0, 1.0 / np.sqrt(np.where(var < 1e-30, 1.0, var)))
    return (X - mean) * inv


# ---------------------------------------------------------------------------------------------
# dense <-> pattern helpers
# ---------------------------------------------------------------------------------------------

def dense_to_csc_values(T_dense, indptr, indices):
    cols = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
    return T_dense[indices, cols]


def dense_to_csr_values(T_dense, indptr, indices):
    rows = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
    return T_dense[rows, indices]


# ---------------------------------------------------------------------------------------------
# searchlight template loop (csrc/ha_template.c:14-114, each ha_procrustes -> searchlight solve)
# ---------------------------------------------------------------------------------------------

def searchlight_template(dms, idx, off, dists, radius, reflection=True, scaling=False, zscore_common=True,
                         level2_iter=1):
    """Sequential running-average template plus leave-one-out passes; aligned = X @ T_searchlight."""
    ns = len(dms)

    def solve(X, Y):
        return searchlight_procrustes_dense(X, Y, idx, off, dists, radius, reflection, scaling)

    common = dms[0].copy()
    aligned = [dms[0].copy()] + [None] * (ns - 1)
    for s in range(1, ns):  # csrc/ha_template.c:39-59
        aligned[s] = dms[s] @ solve(dms[s], common)
        if zscore_common:
            aligned[s] = zscore_columns(aligned[s])
        common = (common + aligned[s]) * 0.5
        if zscore_common:
            common = zscore_columns(common)
    for _ in range(level2_iter):  # csrc/ha_template.c:62-89
        total = aligned[0].copy()
        for s in range(1, ns):
            total = total + aligned[s]
        for s in range(ns):
            ref = (total - aligned[s]) * (1.0 / (ns - 1))
            if zscore_common:
                ref = zscore_columns(ref)
            aligned[s] = dms[s] @ solve(dms[s], ref)
    tpl = aligned[0].copy()  # csrc/ha_template.c:92-103
    for s in range(1, ns):
        tpl = tpl + aligned[s]
    return zscore_columns(tpl) if zscore_common else tpl * (1.0 / ns)
