"""Python entry points of the B200 backend, shaped like the reference ctypes wrapper.

``searchlight_procrustes`` keeps the signature, argument meaning and error
behaviour of the reference's ``hyperalignment_c.searchlight_procrustes``
(hyperalignment_c.py:112-223): Fortran-order float64 X/Y, flattened
searchlights, a zero-initialised dense ``nv x nv`` result from one C call,
``RuntimeError`` on a non-zero return code.  The only backend accepted here is
``"b200"`` (enum value 4); the reference's CPU/Metal/CUDA backends live in the
reference library.

The sparse (CSC) and ridge calls take scipy-compatible CSC arrays whose pattern
is the union of searchlight blocks (``sparse_pattern``, bit-exact to the
reference's ``ha_sparse_init``).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

_BACKENDS = {"b200": L.BACKEND_B200}


def _flatten(sls, dists):
    sizes = np.array([len(s) for s in sls], dtype=np.int32)
    offsets = np.zeros(len(sls) + 1, dtype=np.int32)
    np.cumsum(sizes, out=offsets[1:])
    idx = np.ascontiguousarray(np.concatenate(sls).astype(np.int32))
    d = None if dists is None else np.ascontiguousarray(np.concatenate(dists).astype(np.float64))
    if d is not None and d.size != idx.size:
        raise ValueError("dists must hold one distance per searchlight member")
    return idx, offsets, d


def _check_xy(X, Y):
    """X and Y as Fortran-order float64 of one shape (the library reads nt x nv of each)."""
    X = np.asfortranarray(X, dtype=np.float64)
    Y = np.asfortranarray(Y, dtype=np.float64)
    if X.ndim != 2 or X.shape != Y.shape:
        raise ValueError(f"X and Y must be 2-D arrays of one shape, got {X.shape} and {Y.shape}")
    return X, Y


def _check_csc(indptr, indices, data, nv):
    """The CSC arrays the library reads (indptr, indices) and accumulates into (data, in place)."""
    indptr = np.ascontiguousarray(indptr, dtype=np.int32)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    if indptr.shape != (nv + 1,) or indptr[0] != 0 or indptr[-1] != indices.size:
        raise ValueError("indptr must hold nv + 1 entries from 0 to len(indices)")
    if not isinstance(data, np.ndarray) or data.dtype != np.float64 or not data.flags.c_contiguous \
            or not data.flags.writeable or data.shape != (indices.size,):
        raise ValueError("data must be a writable C-contiguous float64 array of len(indices) entries")
    return indptr, indices


def _check_weights(weights, sls):
    """Per-searchlight weight arrays (or any list of arrays whose concatenation is the flat
    weights): one float64 weight per searchlight member, in searchlight order."""
    if weights is None:
        return None
    w = np.ascontiguousarray(np.concatenate([np.ravel(a) for a in weights]).astype(np.float64))
    if w.size != sum(len(sl) for sl in sls):
        raise ValueError("weights must hold one value per searchlight member")
    return w


def _init():
    lib = L.lib()
    rc = lib.ha_b200_init()
    if rc != 0:
        raise RuntimeError("ha_b200_init() failed. Is an sm_100 (B200) GPU present?")
    return lib


def searchlight_procrustes(X, Y, sls, dists, radius, backend="b200", reflection=True, scaling=False,
                           n_jobs=1, T_out=None):
    """Searchlight Procrustes; returns the dense ``nv x nv`` float64 transformation.

    Same contract as the reference wrapper (hyperalignment_c.py:112-143).  If
    ``T_out`` is given it is accumulated into (the C call's ``+=`` contract) and
    returned; otherwise a zero matrix is allocated.
    """
    if backend not in _BACKENDS:
        raise ValueError(f"Unknown backend '{backend}'. Choose from: {list(_BACKENDS.keys())}")
    X, Y = _check_xy(X, Y)
    idx, offsets, d = _flatten(sls, dists)
    lib = _init()
    if n_jobs > 0:
        lib.ha_set_num_threads(n_jobs)
    nt, nv = X.shape
    if T_out is None:
        T_out = np.zeros((nv, nv), dtype=np.float64)
    elif T_out.dtype != np.float64 or not T_out.flags.c_contiguous or T_out.shape != (nv, nv):
        raise ValueError("T_out must be a C-contiguous float64 (nv, nv) array")
    rc = lib.ha_searchlight_procrustes_dense(
        L.dptr(X), L.dptr(Y), nt, nv, L.iptr(idx), L.iptr(offsets), L.dptr(d), len(sls), float(radius),
        L.dptr(T_out), bool(reflection), bool(scaling), _BACKENDS[backend], True)
    if rc != 0:
        raise RuntimeError(f"ha_searchlight_procrustes_dense failed with error code {rc}")
    return T_out


def searchlight_weights(sls, dists=None, radius=None, nv=None):
    """Flat weights (one per searchlight member), the reference's rule, computed by the library."""
    lib = L.lib()
    idx, offsets, d = _flatten(sls, dists)
    if nv is None:
        nv = int(idx.max()) + 1
    out = np.empty(idx.size, dtype=np.float64)
    L.check(lib.ha_searchlight_weights_b200(L.iptr(idx), L.iptr(offsets), L.dptr(d), len(sls),
                                            float(radius or 0.0), nv, L.dptr(out)), "ha_searchlight_weights_b200")
    return out


def sparse_pattern(sls, nv):
    """CSC pattern (indptr, indices) of the union of ``sl x sl`` blocks, built on the GPU."""
    lib = _init()
    idx, offsets, _ = _flatten(sls, None)
    indptr = np.empty(nv + 1, dtype=np.int32)
    nnz = __import__("ctypes").c_int64(0)
    L.check(lib.ha_sparse_pattern_b200(L.iptr(idx), L.iptr(offsets), len(sls), nv, L.iptr(indptr), None, 0,
                                       __import__("ctypes").byref(nnz)), "ha_sparse_pattern_b200")
    indices = np.empty(nnz.value, dtype=np.int32)
    L.check(lib.ha_sparse_pattern_b200(L.iptr(idx), L.iptr(offsets), len(sls), nv, L.iptr(indptr),
                                       L.iptr(indices), nnz.value, __import__("ctypes").byref(nnz)),
            "ha_sparse_pattern_b200")
    return indptr, indices


def searchlight_procrustes_csc(X, Y, sls, indptr, indices, data, weights=None, reflection=True, scaling=False):
    """Sparse-output searchlight Procrustes: accumulates into ``data`` (CSC, pattern ``indptr``/``indices``)."""
    X, Y = _check_xy(X, Y)
    nt, nv = X.shape
    indptr, indices = _check_csc(indptr, indices, data, nv)
    w = _check_weights(weights, sls)
    lib = _init()
    idx, offsets, _ = _flatten(sls, None)
    L.check(lib.ha_searchlight_procrustes_csc_b200(
        L.dptr(X), L.dptr(Y), nt, nv, L.iptr(idx), L.iptr(offsets), len(sls), L.dptr(w), L.iptr(indptr),
        L.iptr(indices), int(indices.size), L.dptr(data), bool(reflection), bool(scaling), True),
        "ha_searchlight_procrustes_csc_b200")
    return data


def searchlight_ridge_csc(X, Y, sls, indptr, indices, data, alpha, weights=None):
    """Sparse-output searchlight ridge (float64): accumulates into ``data``."""
    X, Y = _check_xy(X, Y)
    nt, nv = X.shape
    indptr, indices = _check_csc(indptr, indices, data, nv)
    w = _check_weights(weights, sls)
    lib = _init()
    idx, offsets, _ = _flatten(sls, None)
    L.check(lib.ha_searchlight_ridge_csc_b200(
        L.dptr(X), L.dptr(Y), nt, nv, L.iptr(idx), L.iptr(offsets), len(sls), L.dptr(w), L.iptr(indptr),
        L.iptr(indices), int(indices.size), L.dptr(data), float(alpha), True), "ha_searchlight_ridge_csc_b200")
    return data


def searchlight_ridge_grid(X, Y, sls, indptr, indices, data, alphas, npcs, train_li, test_li, weights=None,
                           return_costs=False):
    """Searchlight ridge grid search with CV ensembles (float64): the winner's model-averaged
    betas of every searchlight accumulate into ``data`` (CSC); returns the winning grid index per
    searchlight (g = alpha index * len(npcs) + PC index), and the cost grid when asked."""
    X, Y = _check_xy(X, Y)
    nt, nv = X.shape
    indptr, indices = _check_csc(indptr, indices, data, nv)
    w = _check_weights(weights, sls)
    lib = _init()
    idx, offsets, _ = _flatten(sls, None)
    al = np.ascontiguousarray(alphas, dtype=np.float64)
    pc = np.ascontiguousarray(npcs, dtype=np.int32)
    tr, te = L.IndexLists(train_li), L.IndexLists(test_li)
    if len(tr) != len(te):
        raise ValueError("train and test lists differ in length")
    best = np.zeros(len(sls), dtype=np.int32)
    costs = np.zeros((len(sls), al.size, pc.size)) if return_costs else None
    L.check(lib.ha_searchlight_ridge_grid_b200(
        L.dptr(X), L.dptr(Y), nt, nv, L.iptr(idx), L.iptr(offsets), len(sls), L.dptr(w), L.iptr(indptr),
        L.iptr(indices), int(indices.size), L.dptr(data), L.dptr(al), al.size, L.iptr(pc), pc.size, tr.ptrs, te.ptrs,
        L.iptr(tr.sizes), L.iptr(te.sizes), len(tr), L.iptr(best), L.dptr(costs), True),
        "ha_searchlight_ridge_grid_b200")
    return (best, costs) if return_costs else best


def ensemble_indices(nt, n_perms, n_folds, blocksize, buffersize, seed, mask=None):
    """CV split indices with the reference's draws: (train_li, test_li), lists of int32 arrays."""
    lib = L.lib()
    ns = n_perms * n_folds
    train = np.zeros((ns, nt), dtype=np.int32)
    test = np.zeros((ns, nt), dtype=np.int32)
    sizes = np.zeros(ns, dtype=np.int32)
    mk = None
    if mask is not None:
        mk = (ctypes.c_bool * nt)(*[bool(m) for m in mask])
    L.check(lib.ha_ensemble_indices_b200(nt, n_perms, n_folds, blocksize, buffersize, ctypes.c_uint64(seed), mk,
                                         L.iptr(train), L.iptr(test), L.iptr(sizes)), "ha_ensemble_indices_b200")
    return [train[k].copy() for k in range(ns)], [test[k, :sizes[k]].copy() for k in range(ns)]


def cleanup():
    L.lib().ha_b200_cleanup()


def searchlight_template(dms, sls, dists, radius, reflection=True, scaling=False, zscore_common=True,
                         level2_iter=1):
    """Searchlight Procrustes template of subjects ``dms`` (list of nt x nv arrays), on the GPU.

    The loop of the reference's ``ha_template_procrustes`` (csrc/ha_template.c:14-114) with each
    whole-matrix Procrustes replaced by a searchlight solve; returns the nt x nv template.
    """
    ns = len(dms)
    nt, nv = dms[0].shape
    stack = np.empty((ns, nv, nt), dtype=np.float64)  # each subject column-major
    for s, D in enumerate(dms):
        stack[s] = np.asarray(D, dtype=np.float64).T  # raises if a subject's shape differs
    idx, offsets, d = _flatten(sls, dists)
    lib = _init()
    out = np.empty((nv, nt), dtype=np.float64)
    L.check(lib.ha_searchlight_template_b200(
        L.dptr(stack), ns, nt, nv, L.iptr(idx), L.iptr(offsets), L.dptr(d), len(sls), float(radius),
        bool(reflection), bool(scaling), bool(zscore_common), int(level2_iter), L.dptr(out)),
        "ha_searchlight_template_b200")
    return np.ascontiguousarray(out.T)


def searchlight_pca_template(dms, sls, dists, radius, n_jobs=1, tpl_kind="pca"):
    """Searchlight PCA template of subjects ``dms`` (list of nt x nv arrays), on the GPU.

    Same arguments and result as the Python package's ``searchlight_template(dms, sls, dists,
    radius, n_jobs=1, tpl_kind="pca")`` (src/hyperalignment/searchlight.py:215-236); ``n_jobs``
    is accepted and ignored (every searchlight runs on the GPU).  Needs len(sl) <= nt and
    min(nt, len(dms) * len(sl)) <= 512 for every searchlight.
    """
    if tpl_kind != "pca":
        raise ValueError(f"tpl_kind {tpl_kind!r}: only 'pca' runs here (the Procrustes loop is searchlight_template)")
    ns = len(dms)
    nt, nv = np.shape(dms[0])
    stack = np.empty((ns, nv, nt), dtype=np.float64)  # each subject column-major
    for s, D in enumerate(dms):
        stack[s] = np.asarray(D, dtype=np.float64).T
    idx, offsets, d = _flatten(sls, dists)
    lib = _init()
    out = np.empty((nv, nt), dtype=np.float64)
    L.check(lib.ha_searchlight_pca_template_b200(
        L.dptr(stack), ns, nt, nv, L.iptr(idx), L.iptr(offsets), L.dptr(d), len(sls), float(radius), L.dptr(out)),
        "ha_searchlight_pca_template_b200")
    return np.ascontiguousarray(out.T)
