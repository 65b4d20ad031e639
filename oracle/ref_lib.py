"""ctypes binding of the compiled reference library, oracle/_ref/libhyperalignment.so.

TEST INFRASTRUCTURE ONLY (checker and CPU baseline; see oracle/Makefile for how
the reference sources are compiled).  Struct layouts follow csrc/ha_common.h:45-87;
function signatures follow csrc/ha_searchlight.h, csrc/ha_sparse.h,
csrc/ha_procrustes.h, csrc/ha_ridge.h and csrc/ha_ensemble.h.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libhyperalignment.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int32_p = ctypes.POINTER(ctypes.c_int32)


class TMat(ctypes.Structure):  # csrc/ha_common.h:45-49
    _fields_ = [("data", c_double_p), ("rows", ctypes.c_int32), ("cols", ctypes.c_int32)]


class TSparseCSC(ctypes.Structure):  # csrc/ha_common.h:52-59
    _fields_ = [("data", c_double_p), ("indices", c_int32_p), ("indptr", c_int32_p),
                ("rows", ctypes.c_int32), ("cols", ctypes.c_int32), ("nnz", ctypes.c_int64)]


class TSearchlights(ctypes.Structure):  # csrc/ha_common.h:62-68
    _fields_ = [("indices", ctypes.POINTER(c_int32_p)), ("dists", ctypes.POINTER(c_double_p)),
                ("sizes", c_int32_p), ("count", ctypes.c_int32), ("radius", ctypes.c_double)]


_lib = None
REF_CUDA_LIB = os.path.join(HERE, "_ref_cuda", "libhyperalignment_cuda.so")
_cuda_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def cuda_available() -> bool:
    """The reference built with its CUDA arm (make -C oracle cuda) is present."""
    return os.path.exists(REF_CUDA_LIB)


def cuda_lib():
    """The reference library with its own GPU arm (csrc/ha_cuda.cu, cuBLAS + cuSOLVER) compiled for
    sm_100a: the dense entry point with backend 3, and ha_cuda_init / cleanup / available
    (csrc/ha_cuda.h:32-42)."""
    global _cuda_lib
    if _cuda_lib is None:
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        h = ctypes.CDLL(REF_CUDA_LIB)
        h.ha_searchlight_procrustes_dense.restype = ctypes.c_int
        h.ha_searchlight_procrustes_dense.argtypes = [
            c_double_p, c_double_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_double_p,
            ctypes.c_int32, ctypes.c_double, c_double_p, ctypes.c_bool, ctypes.c_bool, ctypes.c_int, ctypes.c_bool]
        h.ha_cuda_init.restype = ctypes.c_int
        h.ha_cuda_init.argtypes = []
        h.ha_cuda_cleanup.restype = None
        h.ha_cuda_cleanup.argtypes = []
        h.ha_cuda_available.restype = ctypes.c_bool
        h.ha_cuda_available.argtypes = []
        h.ha_set_num_threads.restype = None
        h.ha_set_num_threads.argtypes = [ctypes.c_int]
        _cuda_lib = h
    return _cuda_lib


def lib():
    global _lib
    if _lib is None:
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        h = ctypes.CDLL(REF_LIB)
        h.ha_searchlight_procrustes_dense.restype = ctypes.c_int
        h.ha_searchlight_procrustes_dense.argtypes = [
            c_double_p, c_double_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_double_p,
            ctypes.c_int32, ctypes.c_double, c_double_p, ctypes.c_bool, ctypes.c_bool, ctypes.c_int, ctypes.c_bool]
        h.ha_set_num_threads.restype = None
        h.ha_set_num_threads.argtypes = [ctypes.c_int]
        h.ha_get_num_threads.restype = ctypes.c_int
        h.ha_sparse_init.restype = ctypes.POINTER(TSparseCSC)
        h.ha_sparse_init.argtypes = [ctypes.POINTER(TSearchlights), ctypes.c_int32]
        h.ha_sparse_scatter_add.restype = None
        h.ha_sparse_scatter_add.argtypes = [ctypes.POINTER(TSparseCSC), c_int32_p, c_int32_p, ctypes.c_int32,
                                            ctypes.c_int32, c_double_p, c_double_p]
        h.ha_searchlight_weights.restype = ctypes.c_int
        h.ha_searchlight_weights.argtypes = [ctypes.POINTER(TSearchlights), ctypes.POINTER(c_double_p)]
        h.ha_searchlight_procrustes.restype = ctypes.c_int
        h.ha_searchlight_procrustes.argtypes = [
            ctypes.POINTER(TMat), ctypes.POINTER(TMat), ctypes.POINTER(TSearchlights), ctypes.POINTER(TSearchlights),
            ctypes.POINTER(TSparseCSC), ctypes.POINTER(c_double_p), ctypes.c_bool, ctypes.c_bool, ctypes.c_int]
        h.ha_searchlight_ridge.restype = ctypes.c_int
        h.ha_searchlight_ridge.argtypes = [
            ctypes.POINTER(TMat), ctypes.POINTER(TMat), ctypes.POINTER(TSearchlights), ctypes.POINTER(TSearchlights),
            ctypes.POINTER(TSparseCSC), ctypes.POINTER(c_double_p), ctypes.c_double]
        h.ha_procrustes.restype = ctypes.c_int
        h.ha_procrustes.argtypes = [ctypes.POINTER(TMat), ctypes.POINTER(TMat), ctypes.POINTER(TMat), ctypes.c_bool,
                                    ctypes.c_bool]
        h.ha_ridge.restype = ctypes.c_int
        h.ha_ridge.argtypes = [ctypes.POINTER(TMat), ctypes.POINTER(TMat), ctypes.c_double, ctypes.POINTER(TMat)]
        h.ha_ridge_grid.restype = ctypes.c_int  # csrc/ha_ridge.h
        h.ha_ridge_grid.argtypes = [ctypes.POINTER(TMat), c_double_p, c_double_p, ctypes.c_int32, c_int32_p,
                                    ctypes.c_int32, c_int32_p, ctypes.c_int32, c_double_p]
        h.ha_ensemble_ridge.restype = ctypes.c_int
        h.ha_ensemble_ridge.argtypes = [ctypes.POINTER(TMat), c_double_p, c_double_p, ctypes.c_int32, c_int32_p,
                                        ctypes.c_int32, ctypes.POINTER(c_int32_p), ctypes.POINTER(c_int32_p),
                                        c_int32_p, c_int32_p, ctypes.c_int32, c_double_p, c_double_p, c_double_p,
                                        c_double_p, c_int32_p]
        h.ha_ensemble_indices.restype = ctypes.c_int  # csrc/ha_ensemble.h
        h.ha_ensemble_indices.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_bool),
                                          ctypes.POINTER(ctypes.POINTER(c_int32_p)),
                                          ctypes.POINTER(ctypes.POINTER(c_int32_p)),
                                          ctypes.POINTER(c_int32_p), ctypes.POINTER(c_int32_p), c_int32_p]
        h.ha_ensemble_indices_free.restype = None
        h.ha_ensemble_indices_free.argtypes = [ctypes.POINTER(c_int32_p), ctypes.POINTER(c_int32_p), c_int32_p,
                                               c_int32_p, ctypes.c_int32]
        _lib = h
        # one BLAS thread per OpenMP thread (the reference parallelises over searchlights)
        import glob
        import scipy
        libs = os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs")
        for path in glob.glob(os.path.join(libs, "libscipy_openblas*.so")):
            ob = ctypes.CDLL(path)
            fn = getattr(ob, "scipy_openblas_set_num_threads", None)
            if fn is not None:
                fn.argtypes = [ctypes.c_int]
                fn(1)
    return _lib


def _dp(a):
    return a.ctypes.data_as(c_double_p)


def _ip(a):
    return a.ctypes.data_as(c_int32_p)


def set_threads(n: int) -> None:
    lib().ha_set_num_threads(int(n))


def procrustes_dense(X, Y, idx, off, dists, radius, reflection=True, scaling=False, backend=0, threads=None):
    """Reference ha_searchlight_procrustes_dense (cpu64 = 0, cpu32 = 1), column-major input like the wrapper."""
    h = lib()
    if threads is not None:
        h.ha_set_num_threads(int(threads))
    Xf = np.asfortranarray(X, dtype=np.float64)
    Yf = np.asfortranarray(Y, dtype=np.float64)
    nt, nv = Xf.shape
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    off = np.ascontiguousarray(off, dtype=np.int32)
    d = None if dists is None else np.ascontiguousarray(dists, dtype=np.float64)
    T = np.zeros((nv, nv), dtype=np.float64)
    rc = h.ha_searchlight_procrustes_dense(_dp(Xf), _dp(Yf), nt, nv, _ip(idx), _ip(off),
                                           None if d is None else _dp(d), len(off) - 1, float(radius), _dp(T),
                                           bool(reflection), bool(scaling), int(backend), True)
    if rc != 0:
        raise RuntimeError(f"reference ha_searchlight_procrustes_dense rc={rc}")
    return T


def template_procrustes(dms, reflection=True, scaling=False, zscore_common=True, level2_iter=1):
    """Reference ha_template_procrustes (csrc/ha_template.c:14-114): the whole-matrix Procrustes
    template (row-major nt x nv subjects)."""
    h = lib()
    mats = [np.ascontiguousarray(d, dtype=np.float64) for d in dms]
    nt, nv = mats[0].shape
    tms = [TMat(_dp(m), nt, nv) for m in mats]
    arr = (ctypes.POINTER(TMat) * len(tms))(*[ctypes.pointer(t) for t in tms])
    out = np.zeros((nt, nv))
    tout = TMat(_dp(out), nt, nv)
    h.ha_template_procrustes.restype = ctypes.c_int
    h.ha_template_procrustes.argtypes = [ctypes.POINTER(ctypes.POINTER(TMat)), ctypes.c_int32, ctypes.c_bool,
                                         ctypes.c_bool, ctypes.c_bool, ctypes.c_int32, ctypes.POINTER(TMat)]
    rc = h.ha_template_procrustes(arr, len(tms), bool(reflection), bool(scaling), bool(zscore_common),
                                  int(level2_iter), ctypes.byref(tout))
    if rc != 0:
        raise RuntimeError(f"reference ha_template_procrustes rc={rc}")
    return out


class _Sls:
    """Keeps the ctypes arrays of a TSearchlights alive."""

    def __init__(self, idx, off, dists=None, radius=0.0):
        count = len(off) - 1
        self.rows = [np.ascontiguousarray(idx[off[s]:off[s + 1]], dtype=np.int32) for s in range(count)]
        self.sizes = np.array([r.size for r in self.rows], dtype=np.int32)
        self.ptrs = (c_int32_p * count)(*[_ip(r) for r in self.rows])
        self.dists = None
        dptrs = None
        if dists is not None:
            self.dists = [np.ascontiguousarray(dists[off[s]:off[s + 1]], dtype=np.float64) for s in range(count)]
            dptrs = (c_double_p * count)(*[_dp(d) for d in self.dists])
        self.dptrs = dptrs
        self.st = TSearchlights(self.ptrs, dptrs if dptrs is not None else None, _ip(self.sizes), count, float(radius))


def sparse_init(idx, off, nv):
    """Reference ha_sparse_init: returns (indptr int32, indices int32)."""
    h = lib()
    sls = _Sls(idx, off)
    m = h.ha_sparse_init(ctypes.byref(sls.st), int(nv))
    if not m:
        raise RuntimeError("ha_sparse_init returned NULL")
    mat = m.contents
    indptr = np.ctypeslib.as_array(mat.indptr, shape=(nv + 1,)).copy()
    indices = np.ctypeslib.as_array(mat.indices, shape=(mat.nnz,)).copy() if mat.nnz > 0 else np.zeros(0, np.int32)
    return indptr, indices


def searchlight_weights(idx, off, dists, radius):
    h = lib()
    sls = _Sls(idx, off, dists, radius)
    count = len(off) - 1
    out = (c_double_p * count)()
    rc = h.ha_searchlight_weights(ctypes.byref(sls.st), out)
    if rc != 0:
        raise RuntimeError(f"ha_searchlight_weights rc={rc}")
    return np.concatenate([np.ctypeslib.as_array(out[s], shape=(int(sls.sizes[s]),)).copy() for s in range(count)])


def _csc_struct(indptr, indices, data, nv):
    return TSparseCSC(_dp(data), _ip(indices), _ip(indptr), nv, nv, len(indices))


def searchlight_procrustes_csc(X, Y, idx, off, indptr, indices, weights=None, reflection=True, scaling=False,
                               backend=0, threads=None):
    """Reference sparse-API ha_searchlight_procrustes (row-major TMat input); returns CSC data."""
    h = lib()
    if threads is not None:
        h.ha_set_num_threads(int(threads))
    Xc = np.ascontiguousarray(X, dtype=np.float64)
    Yc = np.ascontiguousarray(Y, dtype=np.float64)
    nt, nv = Xc.shape
    indptr = np.ascontiguousarray(indptr, dtype=np.int32)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    data = np.zeros(len(indices), dtype=np.float64)
    mat = _csc_struct(indptr, indices, data, nv)
    tx, ty = TMat(_dp(Xc), nt, nv), TMat(_dp(Yc), nt, nv)
    sls = _Sls(idx, off)
    wp = None
    if weights is not None:
        ws = [np.ascontiguousarray(weights[off[s]:off[s + 1]], dtype=np.float64) for s in range(len(off) - 1)]
        wp = (c_double_p * len(ws))(*[_dp(w) for w in ws])
        keep = ws  # noqa: F841
    rc = h.ha_searchlight_procrustes(ctypes.byref(tx), ctypes.byref(ty), ctypes.byref(sls.st), None,
                                     ctypes.byref(mat), wp, bool(reflection), bool(scaling), int(backend))
    if rc != 0:
        raise RuntimeError(f"reference ha_searchlight_procrustes rc={rc}")
    return data


def searchlight_ridge_csc(X, Y, idx, off, indptr, indices, alpha, weights=None, threads=None):
    h = lib()
    if threads is not None:
        h.ha_set_num_threads(int(threads))
    Xc = np.ascontiguousarray(X, dtype=np.float64)
    Yc = np.ascontiguousarray(Y, dtype=np.float64)
    nt, nv = Xc.shape
    indptr = np.ascontiguousarray(indptr, dtype=np.int32)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    data = np.zeros(len(indices), dtype=np.float64)
    mat = _csc_struct(indptr, indices, data, nv)
    tx, ty = TMat(_dp(Xc), nt, nv), TMat(_dp(Yc), nt, nv)
    sls = _Sls(idx, off)
    wp = None
    if weights is not None:
        ws = [np.ascontiguousarray(weights[off[s]:off[s + 1]], dtype=np.float64) for s in range(len(off) - 1)]
        wp = (c_double_p * len(ws))(*[_dp(w) for w in ws])
        keep = ws  # noqa: F841
    rc = h.ha_searchlight_ridge(ctypes.byref(tx), ctypes.byref(ty), ctypes.byref(sls.st), None, ctypes.byref(mat),
                                wp, float(alpha))
    if rc != 0:
        raise RuntimeError(f"reference ha_searchlight_ridge rc={rc}")
    return data


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def ridge_grid(X, y, alphas, npcs, train_idx=None):
    """ha_ridge_grid (csrc/ha_ridge.c:97-227): betas[v, a, p] for one target vector y."""
    h = lib()
    Xc = np.ascontiguousarray(X, dtype=np.float64)
    yc = np.ascontiguousarray(y, dtype=np.float64)
    al = np.ascontiguousarray(alphas, dtype=np.float64)
    npc = _i32(npcs)
    out = np.zeros((Xc.shape[1], al.size, npc.size))
    tx = TMat(_dp(Xc), Xc.shape[0], Xc.shape[1])
    tr = None if train_idx is None else _i32(train_idx)
    rc = h.ha_ridge_grid(ctypes.byref(tx), _dp(yc), _dp(al), al.size, _ip(npc), npc.size,
                         None if tr is None else _ip(tr), 0 if tr is None else tr.size, _dp(out))
    if rc != 0:
        raise RuntimeError(f"reference ha_ridge_grid rc={rc}")
    return out


def ensemble_ridge(X, y, alphas, npcs, train_li, test_li):
    """ha_ensemble_ridge (csrc/ha_ridge.c:229-345) for one target: (weights, pred, r2, alpha, npc)."""
    h = lib()
    Xc = np.ascontiguousarray(X, dtype=np.float64)
    yc = np.ascontiguousarray(y, dtype=np.float64)
    al = np.ascontiguousarray(alphas, dtype=np.float64)
    npc = _i32(npcs)
    trs = [_i32(t) for t in train_li]
    tes = [_i32(t) if len(t) else np.zeros(1, dtype=np.int32) for t in test_li]
    trp = (c_int32_p * len(trs))(*[_ip(t) for t in trs])
    tep = (c_int32_p * len(tes))(*[_ip(t) for t in tes])
    trn = _i32([t.size for t in trs])
    ten = _i32([len(t) for t in test_li])
    nt, nv = Xc.shape
    w = np.zeros(nv)
    pred = np.zeros(nt)
    r2, alpha = ctypes.c_double(), ctypes.c_double()
    npc_out = ctypes.c_int32()
    tx = TMat(_dp(Xc), nt, nv)
    rc = h.ha_ensemble_ridge(ctypes.byref(tx), _dp(yc), _dp(al), al.size, _ip(npc), npc.size, trp, tep, _ip(trn),
                             _ip(ten), len(trs), _dp(w), _dp(pred), ctypes.byref(r2), ctypes.byref(alpha),
                             ctypes.byref(npc_out))
    if rc != 0:
        raise RuntimeError(f"reference ha_ensemble_ridge rc={rc}")
    return w, pred, r2.value, alpha.value, npc_out.value


def ensemble_indices(nt, n_perms, n_folds, blocksize, buffersize, seed, mask=None):
    """ha_ensemble_indices (csrc/ha_ensemble.c:58-249): (train_li, test_li) as numpy arrays."""
    h = lib()
    tr = ctypes.POINTER(c_int32_p)()
    te = ctypes.POINTER(c_int32_p)()
    trn, ten = c_int32_p(), c_int32_p()
    ns = ctypes.c_int32()
    mk = None
    if mask is not None:
        mk = (ctypes.c_bool * nt)(*[bool(m) for m in mask])
    rc = h.ha_ensemble_indices(nt, n_perms, n_folds, blocksize, buffersize, ctypes.c_uint64(seed), mk,
                               ctypes.byref(tr), ctypes.byref(te), ctypes.byref(trn), ctypes.byref(ten),
                               ctypes.byref(ns))
    if rc != 0:
        raise RuntimeError(f"reference ha_ensemble_indices rc={rc}")
    train_li = [np.ctypeslib.as_array(tr[k], shape=(trn[k],)).copy() for k in range(ns.value)]
    test_li = [np.ctypeslib.as_array(te[k], shape=(ten[k],)).copy() if ten[k] else np.zeros(0, dtype=np.int32)
               for k in range(ns.value)]
    h.ha_ensemble_indices_free(tr, te, trn, ten, ns.value)
    return train_li, test_li
