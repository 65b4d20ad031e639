"""Device-resident plan: one searchlight geometry, many solves (include/hyperalignment_b200.h).

Device memory and streams are whatever the caller owns; this wrapper takes raw
device pointers (ints), e.g. ``tensor.data_ptr()`` of CUDA tensors, and a raw
``cudaStream_t`` handle (``torch.cuda.current_stream().cuda_stream``) or 0.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L


class Plan:
    def __init__(self, nt, nv, indices, offsets, dists=None, radius=0.0, weights=None):
        self.lib = L.lib()
        L.check(self.lib.ha_b200_init(), "ha_b200_init")
        self.nt, self.nv = int(nt), int(nv)
        self.indices = np.ascontiguousarray(indices, dtype=np.int32)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        self.count = int(self.offsets.size - 1)
        d = None if dists is None else np.ascontiguousarray(dists, dtype=np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        h = ctypes.c_void_p()
        L.check(self.lib.ha_b200_plan_create(self.nt, self.nv, L.iptr(self.indices), L.iptr(self.offsets), L.dptr(d),
                                             self.count, float(radius), L.dptr(w), ctypes.byref(h)),
                "ha_b200_plan_create")
        self.handle = h

    @classmethod
    def from_workload(cls, w, weights=None):
        return cls(w.nt, w.nv, w.sls.indices, w.sls.offsets, w.sls.dists, w.sls.radius, weights)

    @property
    def nnz(self) -> int:
        return int(self.lib.ha_b200_plan_nnz(self.handle))

    def pattern(self):
        indptr = np.empty(self.nv + 1, dtype=np.int64)
        indices = np.empty(self.nnz, dtype=np.int32)
        L.check(self.lib.ha_b200_plan_pattern(self.handle, indptr.ctypes.data_as(L.c_int64_p), L.iptr(indices)),
                "ha_b200_plan_pattern")
        return indptr, indices

    def procrustes_device(self, d_X: int, d_Y: int, d_values: int, reflection=True, scaling=False,
                          solver=L.SOLVER_MIXED, out_kind=L.OUT_CSR, stream: int = 0):
        L.check(self.lib.ha_b200_plan_procrustes_device(self.handle, ctypes.c_void_p(d_X), ctypes.c_void_p(d_Y),
                                                        bool(reflection), bool(scaling), int(solver), int(out_kind),
                                                        ctypes.c_void_p(d_values), ctypes.c_void_p(stream)),
                "ha_b200_plan_procrustes_device")

    def ridge_device(self, d_X: int, d_Y: int, d_values: int, alpha: float, out_kind=L.OUT_CSC, stream: int = 0):
        L.check(self.lib.ha_b200_plan_ridge_device(self.handle, ctypes.c_void_p(d_X), ctypes.c_void_p(d_Y),
                                                   float(alpha), int(out_kind), ctypes.c_void_p(d_values),
                                                   ctypes.c_void_p(stream)), "ha_b200_plan_ridge_device")

    def ridge_grid_device(self, d_X: int, d_Y: int, d_values: int, d_best: int, alphas, npcs, train_li, test_li,
                          d_cost: int = 0, out_kind=L.OUT_CSC, stream: int = 0):
        al = np.ascontiguousarray(alphas, dtype=np.float64)
        pc = np.ascontiguousarray(npcs, dtype=np.int32)
        tr, te = L.IndexLists(train_li), L.IndexLists(test_li)
        L.check(self.lib.ha_b200_plan_ridge_grid_device(
            self.handle, ctypes.c_void_p(d_X), ctypes.c_void_p(d_Y), L.dptr(al), al.size, L.iptr(pc), pc.size,
            tr.ptrs, te.ptrs, L.iptr(tr.sizes), L.iptr(te.sizes), len(tr), out_kind, ctypes.c_void_p(d_values),
            ctypes.c_void_p(d_best), ctypes.c_void_p(d_cost or None), ctypes.c_void_p(stream)),
            "ha_b200_plan_ridge_grid_device")

    def ridge_features_device(self, d_X: int, rows, d_features: int, stream: int = 0):
        r = np.ascontiguousarray(rows, dtype=np.int32)
        L.check(self.lib.ha_b200_plan_ridge_features_device(self.handle, ctypes.c_void_p(d_X), L.iptr(r), r.size,
                                                            ctypes.c_void_p(d_features), ctypes.c_void_p(stream)),
                "ha_b200_plan_ridge_features_device")

    def ridge_learned_device(self, d_X: int, d_Y: int, rows, alphas, npcs, d_params: int, min_prob: float,
                             train_li, test_li, d_values: int, d_choice: int, d_prob: int, out_kind=L.OUT_CSC,
                             stream: int = 0):
        r = np.ascontiguousarray(rows, dtype=np.int32)
        al = np.ascontiguousarray(alphas, dtype=np.float64)
        pc = np.ascontiguousarray(npcs, dtype=np.int32)
        tr, te = L.IndexLists(train_li), L.IndexLists(test_li)
        L.check(self.lib.ha_b200_plan_ridge_learned_device(
            self.handle, ctypes.c_void_p(d_X), ctypes.c_void_p(d_Y), L.iptr(r), r.size, L.dptr(al), al.size,
            L.iptr(pc), pc.size, ctypes.c_void_p(d_params), float(min_prob), tr.ptrs, te.ptrs, L.iptr(tr.sizes),
            L.iptr(te.sizes), len(tr), out_kind, ctypes.c_void_p(d_values), ctypes.c_void_p(d_choice),
            ctypes.c_void_p(d_prob), ctypes.c_void_p(stream)), "ha_b200_plan_ridge_learned_device")

    def aligned_correlation_device(self, d_X: int, d_Y: int, d_values: int, d_r: int, d_aligned: int = 0,
                                   nt: int | None = None, stream: int = 0):
        """Vertex-wise correlation of X @ W with Y (W: this plan's pattern with d_values in CSC order,
        as a kHaB200OutCSC run leaves them; d_values 0 correlates X itself) into d_r (nv float64).
        X and Y (nt x nv, column-major) may be other time points than the plan's, e.g. held-out
        ones: nt defaults to the plan's."""
        ptr, idx = ctypes.c_void_p(), ctypes.c_void_p()
        L.check(self.lib.ha_b200_plan_device_pattern(self.handle, ctypes.byref(ptr), ctypes.byref(idx)),
                "ha_b200_plan_device_pattern")
        L.check(self.lib.ha_b200_aligned_correlation_device(
            ctypes.c_void_p(d_X), ctypes.c_void_p(d_Y), int(self.nt if nt is None else nt), self.nv, ptr, idx,
            ctypes.c_void_p(d_values or None),
            self.nnz, ctypes.c_void_p(d_r), ctypes.c_void_p(d_aligned or None), ctypes.c_void_p(stream)),
            "ha_b200_aligned_correlation_device")

    def stats(self):
        a, b = ctypes.c_int32(), ctypes.c_int32()
        L.check(self.lib.ha_b200_plan_stats(self.handle, ctypes.byref(a), ctypes.byref(b)), "ha_b200_plan_stats")
        ssum, smax = ctypes.c_int64(), ctypes.c_int32()
        L.check(self.lib.ha_b200_plan_sweep_stats(self.handle, ctypes.byref(ssum), ctypes.byref(smax)),
                "ha_b200_plan_sweep_stats")
        return {"n_fp64": a.value, "n_unconverged": b.value, "sweeps_mean": ssum.value / max(1, self.count),
                "sweeps_max": smax.value}

    def searchlight_stats(self, first: int, n: int):
        """Per-searchlight sigma_min, sigma_max, flags and sweeps of the last run (last chunk)."""
        smin, smax = np.empty(n), np.empty(n)
        flags, sweeps = np.empty(n, dtype=np.int32), np.empty(n, dtype=np.int32)
        L.check(self.lib.ha_b200_plan_searchlight_stats(self.handle, first, n, L.dptr(smin), L.dptr(smax),
                                                         L.iptr(flags), L.iptr(sweeps)),
                "ha_b200_plan_searchlight_stats")
        return {"s_min": smin, "s_max": smax, "flags": flags, "sweeps": sweeps}

    def local_transforms(self, first: int, n: int):
        """Unweighted, unscaled T_s of searchlights [first, first+n) from the last run: T_s after a CSR
        run, T_s transposed after a CSC run (the T scratch is column-major then)."""
        sizes = np.diff(self.offsets[first:first + n + 1])
        buf = np.empty(int((sizes.astype(np.int64) ** 2).sum()), dtype=np.float32)
        L.check(self.lib.ha_b200_plan_local_transforms(self.handle, first, n,
                                                        buf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                "ha_b200_plan_local_transforms")
        out, o = [], 0
        for k in sizes:
            out.append(buf[o:o + k * k].reshape(k, k).astype(np.float64))
            o += k * k
        return out

    def tc_layout(self):
        """Tensor-core tile layout per size class: shared memory per CTA (KB), whether it was tuned or
        pinned, and the candidates' measured Gram-launch times (ms; 0 = not timed)."""
        kb = np.zeros(2, dtype=np.int32)
        tuned = ctypes.c_int32()
        ms = np.zeros(6)
        L.check(self.lib.ha_b200_plan_tc_layout(self.handle, L.iptr(kb), ctypes.byref(tuned), L.dptr(ms)),
                "ha_b200_plan_tc_layout")
        return {"smem_kb": [int(x) for x in kb], "tuned": bool(tuned.value),
                "candidates_ms": {"le128_cols": {"110": ms[0], "72": ms[1], "53": ms[2]},
                                  "129_256_cols": {"110": ms[3], "200": ms[4]}}}

    def set_tc_layout(self, smem_kb):
        kb = np.ascontiguousarray(smem_kb, dtype=np.int32)
        L.check(self.lib.ha_b200_plan_set_tc_layout(self.handle, L.iptr(kb)), "ha_b200_plan_set_tc_layout")

    def set_grid_precision(self, bits: int):
        """Arithmetic of ridge_grid_device: 64 (float64, the default) or 32 (the plain FP32 form)."""
        L.check(self.lib.ha_b200_plan_set_grid_precision(self.handle, int(bits)), "ha_b200_plan_set_grid_precision")

    def close(self):
        if self.handle:
            self.lib.ha_b200_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
