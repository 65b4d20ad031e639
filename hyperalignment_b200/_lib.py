"""ctypes binding of ``libha_b200.so`` (declarations in include/hyperalignment_b200.h).

Loading never falls back to anything: if the shared library is missing or
fails to load, :func:`lib` raises.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libha_b200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_int64_p = ctypes.POINTER(ctypes.c_int64)

# name -> (restype, argtypes); every function the header declares.
SIGNATURES = {
    "ha_b200_init": (ctypes.c_int, []),
    "ha_b200_cleanup": (None, []),
    "ha_b200_available": (ctypes.c_bool, []),
    "ha_set_num_threads": (None, [ctypes.c_int]),
    "ha_get_num_threads": (ctypes.c_int, []),
    "ha_searchlight_procrustes_dense": (ctypes.c_int, [
        c_double_p, c_double_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_double_p,
        ctypes.c_int32, ctypes.c_double, c_double_p, ctypes.c_bool, ctypes.c_bool, ctypes.c_int,
        ctypes.c_bool]),
    "ha_searchlight_procrustes_b200": (ctypes.c_int, [
        c_double_p, c_double_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_double_p,
        ctypes.c_int32, ctypes.c_double, c_double_p, ctypes.c_bool, ctypes.c_bool, ctypes.c_bool]),
    "ha_sparse_pattern_b200": (ctypes.c_int, [
        c_int32_p, c_int32_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, ctypes.c_int64,
        c_int64_p]),
    "ha_searchlight_weights_b200": (ctypes.c_int, [
        c_int32_p, c_int32_p, c_double_p, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, c_double_p]),
    "ha_searchlight_procrustes_csc_b200": (ctypes.c_int, [
        c_double_p, c_double_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, ctypes.c_int32,
        c_double_p, c_int32_p, c_int32_p, ctypes.c_int64, c_double_p, ctypes.c_bool, ctypes.c_bool,
        ctypes.c_bool]),
    "ha_searchlight_ridge_csc_b200": (ctypes.c_int, [
        c_double_p, c_double_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, ctypes.c_int32,
        c_double_p, c_int32_p, c_int32_p, ctypes.c_int64, c_double_p, ctypes.c_double, ctypes.c_bool]),
    "ha_searchlight_ridge_grid_b200": (ctypes.c_int, [
        c_double_p, c_double_p, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, ctypes.c_int32,
        c_double_p, c_int32_p, c_int32_p, ctypes.c_int64, c_double_p, c_double_p, ctypes.c_int32, c_int32_p,
        ctypes.c_int32, ctypes.POINTER(c_int32_p), ctypes.POINTER(c_int32_p), c_int32_p, c_int32_p, ctypes.c_int32,
        c_int32_p, c_double_p, ctypes.c_bool]),
    "ha_ensemble_indices_b200": (ctypes.c_int, [
        ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64,
        ctypes.POINTER(ctypes.c_bool), c_int32_p, c_int32_p, c_int32_p]),
    "ha_searchlight_template_b200": (ctypes.c_int, [
        c_double_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_double_p, ctypes.c_int32,
        ctypes.c_double, ctypes.c_bool, ctypes.c_bool, ctypes.c_bool, ctypes.c_int32, c_double_p]),
    "ha_searchlight_pca_template_b200": (ctypes.c_int, [
        c_double_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_double_p, ctypes.c_int32,
        ctypes.c_double, c_double_p]),
    "ha_b200_plan_create": (ctypes.c_int, [
        ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p, c_double_p, ctypes.c_int32, ctypes.c_double,
        c_double_p, ctypes.POINTER(ctypes.c_void_p)]),
    "ha_b200_plan_destroy": (None, [ctypes.c_void_p]),
    "ha_b200_plan_nnz": (ctypes.c_int64, [ctypes.c_void_p]),
    "ha_b200_plan_pattern": (ctypes.c_int, [ctypes.c_void_p, c_int64_p, c_int32_p]),
    "ha_b200_plan_device_pattern": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]),
    "ha_b200_plan_stats": (ctypes.c_int, [ctypes.c_void_p, c_int32_p, c_int32_p]),
    "ha_b200_plan_sweep_stats": (ctypes.c_int, [ctypes.c_void_p, c_int64_p, c_int32_p]),
    "ha_b200_plan_searchlight_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, c_double_p,
                                                      c_double_p, c_int32_p, c_int32_p]),
    "ha_b200_plan_procrustes_device": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_bool, ctypes.c_bool, ctypes.c_int,
        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "ha_b200_plan_ridge_device": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
        ctypes.c_void_p]),
    "ha_b200_plan_ridge_grid_device": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, c_double_p, ctypes.c_int32, c_int32_p, ctypes.c_int32,
        ctypes.POINTER(c_int32_p), ctypes.POINTER(c_int32_p), c_int32_p, c_int32_p, ctypes.c_int32, ctypes.c_int,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ha_b200_plan_local_transforms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, c_float_p]),
    "ha_b200_local_procrustes_noalloc": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, c_int32_p, ctypes.c_int32,
        ctypes.c_void_p, ctypes.c_void_p]),
    "ha_b200_plan_ridge_features_device": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, c_int32_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    "ha_b200_plan_ridge_learned_device": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, c_int32_p, ctypes.c_int32, c_double_p, ctypes.c_int32,
        c_int32_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_float, ctypes.POINTER(c_int32_p),
        ctypes.POINTER(c_int32_p), c_int32_p, c_int32_p, ctypes.c_int32, ctypes.c_int, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ha_b200_mlp_param_count": (ctypes.c_int64, [ctypes.c_int32]),
    "ha_b200_mlp_init": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint64]),
    "ha_b200_mlp_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int32, ctypes.c_void_p, c_float_p]),
    "ha_b200_mlp_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                         ctypes.c_uint64, c_float_p]),
    "ha_b200_mlp_infer": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "ha_b200_set_kernel_timing": (None, [ctypes.c_bool]),
    "ha_b200_kernel_times": (ctypes.c_int, [c_double_p, c_int64_p]),
    "ha_b200_launch_count": (ctypes.c_int64, []),
    "ha_b200_tc_selftest": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_float_p, c_float_p,
                                           c_float_p]),
    "ha_b200_plan_tc_layout": (ctypes.c_int, [ctypes.c_void_p, c_int32_p, c_int32_p, c_double_p]),
    "ha_b200_set_graphs": (None, [ctypes.c_bool]),
    "ha_b200_plan_set_tc_layout": (ctypes.c_int, [ctypes.c_void_p, c_int32_p]),
    "ha_b200_plan_set_grid_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "ha_b200_aligned_correlation_device": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
}

KERNEL_KINDS = ["convert", "colvar", "xcov32", "jacobi32", "formT32", "xcov64", "jacobi64", "formT64", "refine",
                "reflect", "scale", "reduce", "pattern", "ridge", "grid", "mlp", "eval", "tc_xcov", "tc_ns",
                "pca"]

# Error codes and enum values (include/hyperalignment_b200.h, same as the reference's ha_common.h).
SUCCESS, ERROR_ALLOC, ERROR_SVD, ERROR_ARG, ERROR_INTERNAL = 0, -1, -2, -3, -4
BACKEND_B200 = 4
OUT_CSR, OUT_CSC = 0, 1
SOLVER_MIXED, SOLVER_FP32, SOLVER_FP64, SOLVER_TC = 0, 1, 2, 3

_lib = None


def lib() -> ctypes.CDLL:
    """Load ``libha_b200.so`` (raises if it is missing; there is no other implementation)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is not built; run `python -m hyperalignment_b200.build` (needs nvcc)")
        h = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def check(rc: int, what: str) -> None:
    if rc != SUCCESS:
        raise RuntimeError(f"{what} failed with error code {rc}")


def dptr(a):
    return None if a is None else a.ctypes.data_as(c_double_p)


def iptr(a):
    return None if a is None else a.ctypes.data_as(c_int32_p)


class IndexLists:
    """Lists of int32 row arrays as the C ``const int32_t *const *`` + sizes pair (kept alive here)."""

    def __init__(self, lists):
        import numpy as np
        self.arrays = [np.ascontiguousarray(a, dtype=np.int32) for a in lists]
        self.keep = [a if a.size else np.zeros(1, dtype=np.int32) for a in self.arrays]
        self.ptrs = (c_int32_p * len(self.keep))(*[iptr(a) for a in self.keep])
        self.sizes = np.array([a.size for a in self.arrays], dtype=np.int32)

    def __len__(self):
        return len(self.arrays)
