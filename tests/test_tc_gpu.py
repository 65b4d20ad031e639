"""GPU parity of the tensor-core solver (kHaB200SolverTC) through the C ABI.

Tolerances (written per test):
  * one tensor-core product vs float64: relative Frobenius <= 5e-6 (the cross-covariance: three
    BF16 parts, six products; the iteration's Gram and update: two FP16 parts of x 2^12, three
    products; FP32 accumulation over K up to 512)
  * per-searchlight transform T_s vs the float64 oracle: relative Frobenius <= 2e-5 (the
    metric's bound is 1e-4; the three-part split carries FP32 accuracy, measured 1.0e-5 at
    n = 512)
  * dense results vs the reference float64 / float32 CPU backends: relative Frobenius and
    max-abs <= 1e-5
  * repeated runs: bitwise identical
"""

import numpy as np
import pytest

from conftest import golden
from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import workloads as W
from hyperalignment_b200.plan import Plan
from oracle import ha_oracle as O

pytestmark = pytest.mark.gpu

PROD_REL = 5e-6
T_REL_TC = 2e-5
GLOBAL_REL = 1e-5


def relf(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def selftest(hlib, which, n, a, b=None, nt=0):
    out = np.zeros((n, n), dtype=np.float32)
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = None if b is None else np.ascontiguousarray(b, dtype=np.float32)
    fp = L.c_float_p
    rc = hlib.ha_b200_tc_selftest(which, n, nt, a.ctypes.data_as(fp),
                                  None if b is None else b.ctypes.data_as(fp), out.ctypes.data_as(fp))
    assert rc == 0
    return out.astype(np.float64)


@pytest.mark.parametrize("n", [16, 40, 100, 128, 144, 200, 256, 272, 304, 400, 512])
def test_tc_products(gpu, hlib, n):
    """Each product type of the solver on one matrix: X^T X (MN-major A and B), X M (K-major A,
    MN-major B), and the gathered cross-covariance (K-major A and B, K = time).  The iteration's
    operands are in its range (entries of a matrix with singular values about 1, so X^T X and
    X M stay below the FP16 planes' limit); the cross-covariance's inputs have any scale."""
    rng = np.random.default_rng(n)
    X = (rng.standard_normal((n, n)) / np.sqrt(n)).astype(np.float32)
    M = (rng.standard_normal((n, n)) / np.sqrt(n)).astype(np.float32)
    x64, m64 = X.astype(np.float64), M.astype(np.float64)
    assert relf(selftest(hlib, 0, n, X), x64.T @ x64) <= PROD_REL
    assert relf(selftest(hlib, 1, n, X, M), x64 @ m64) <= PROD_REL
    nt = 200 + (n % 3) * 7  # time length not a multiple of 16
    A = rng.standard_normal((n, nt)).astype(np.float32)  # vertex-major: row j = vertex j's series
    B = rng.standard_normal((n, nt)).astype(np.float32)
    got = selftest(hlib, 2, n, A, B, nt=nt)
    assert relf(got, A.astype(np.float64) @ B.astype(np.float64).T) <= PROD_REL


def _device_run(w, solver, refl=True, scal=False, out_kind=L.OUT_CSR):
    import torch
    plan = Plan.from_workload(w)
    dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).cuda()
    dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).cuda()
    vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
    plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), refl, scal, solver, out_kind)
    torch.cuda.synchronize()
    return plan, vals.cpu().numpy()


@pytest.mark.parametrize("lo,hi", [(1, 12), (60, 90), (150, 240), (250, 300), (300, 420), (481, 512)])
def test_tc_local_transforms_vs_fp64(gpu, lo, hi):
    """Per-searchlight T_s of the tensor-core solver against the float64 oracle, across one to four
    128-row tiles and both size classes."""
    nv = 642 if hi <= 240 else 1442
    w = W.small_case(seed=11, nv=nv, nt=max(2 * hi, 40), lo=lo, hi=hi)
    count = min(w.sls.count, 24)
    w.sls = w.sls.subset(np.arange(count))
    plan, _ = _device_run(w, L.SOLVER_TC)
    Ts = plan.local_transforms(0, count)
    worst = 0.0
    for q in range(count):
        sl = w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]
        worst = max(worst, relf(Ts[q], O.procrustes(w.X[:, sl], w.Y[:, sl])))
    assert worst <= T_REL_TC, worst
    assert plan.stats()["n_fp64"] == 0


@pytest.mark.parametrize("key,weighted", [("T_cpu64", True), ("T_cpu64_uniform", False)])
def test_tc_dense_matches_reference_golden(gpu, key, weighted):
    g = golden("small_dense.npz")
    w = W.Workload("golden", g["X"], g["Y"],
                   W.Searchlights(g["idx"], g["off"], g["dists"] if weighted else None, float(g["radius"]),
                                  g["X"].shape[1]), True, False)
    plan, csr = _device_run(w, L.SOLVER_TC)
    indptr, indices = plan.pattern()
    ref = O.dense_to_csr_values(g[key], indptr, indices)
    assert relf(csr, ref) <= GLOBAL_REL
    assert np.abs(csr - ref).max() <= GLOBAL_REL
    if key == "T_cpu64":
        assert relf(csr, O.dense_to_csr_values(g["T_cpu32"], indptr, indices)) <= GLOBAL_REL


def test_tc_scaling_vs_oracle(gpu):
    w = W.small_case(seed=21, nv=642, nt=120, lo=30, hi=80, scaling=True)
    s = w.sls
    plan, csr = _device_run(w, L.SOLVER_TC, scal=True)
    indptr, indices = plan.pattern()
    Tref = O.searchlight_procrustes_dense(w.X, w.Y, s.indices, s.offsets, s.dists, s.radius, True, True)
    assert relf(csr, O.dense_to_csr_values(Tref, indptr, indices)) <= GLOBAL_REL


def test_tc_is_deterministic(gpu):
    w = W.small_case(seed=3, nv=642, nt=60, lo=20, hi=60)
    _, a = _device_run(w, L.SOLVER_TC)
    _, b = _device_run(w, L.SOLVER_TC)
    assert a.tobytes() == b.tobytes()


@pytest.mark.parametrize("out_kind", [L.OUT_CSR, L.OUT_CSC])  # T row-major / column-major in the completion
def test_tc_rank_deficient_searchlights(gpu, out_kind):
    """Exactly singular A keeps zero singular values the iteration cannot grow: the iteration
    stalls and the null spaces are completed (flag 16), keeping T orthogonal; X @ T and T on the
    row space of A are unique and match the oracle."""
    w = W.small_case(seed=9, nv=642, nt=100, lo=30, hi=60)
    mask = W.duplicate_columns(w.X, w.sls, 0.5, np.random.default_rng(1))
    assert mask.sum() > 0
    plan, _ = _device_run(w, L.SOLVER_TC, out_kind=out_kind)
    Ts = plan.local_transforms(0, w.sls.count)
    if out_kind == L.OUT_CSC:  # the T scratch is column-major after a CSC run
        Ts = [t.T for t in Ts]
    worst = 0.0
    for q in np.flatnonzero(mask)[:40]:
        sl = w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]
        Xs = w.X[:, sl]
        Tref = O.procrustes(Xs, w.Y[:, sl])
        worst = max(worst, relf(Xs @ Ts[q], Xs @ Tref))
        _, sv, Vt = np.linalg.svd(Xs.T @ w.Y[:, sl])
        Vp = Vt[sv > sv[0] * 1e-9].T
        worst = max(worst, relf(Ts[q] @ Vp @ Vp.T, Tref @ Vp @ Vp.T))
        assert np.abs(Ts[q].T @ Ts[q] - np.eye(sl.size)).max() < 1e-4
    assert worst <= 1e-4, worst
    # completed searchlights are exactly the singular ones (the generator's mask misses searchlights
    # that hold two copies of one column without the original, so singularity is read off the SVD)
    singular = np.array([
        (lambda s: s[-1] <= s[0] * 1e-10)(np.linalg.svd(
            w.X[:, w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]].T
            @ w.Y[:, w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]], compute_uv=False))
        for q in range(w.sls.count)])
    completed = (plan.searchlight_stats(0, w.sls.count)["flags"] & 16) != 0
    assert not (completed & ~singular).any()
    assert completed.sum() >= singular.sum() // 2


def test_tc_accuracy_at_full_size(gpu):
    """Template workload (10242 searchlights of 100-300): the 150 searchlights that needed the most
    iterations (the worst conditioned: condition numbers up to ~4e5) and 50 others, each within the
    metric's 1e-4 of float64, with no float64 re-solve."""
    w = W.template_procrustes_pair(seed=0)
    plan, _ = _device_run(w, L.SOLVER_TC, scal=True)
    iters = plan.searchlight_stats(0, w.sls.count)["sweeps"]
    rng = np.random.default_rng(7)
    pick = np.unique(np.concatenate([np.argsort(-iters, kind="stable")[:150], rng.choice(w.sls.count, 50, replace=False)]))
    worst = 0.0
    for q in pick:
        T = plan.local_transforms(int(q), 1)[0]
        sl = w.sls.indices[w.sls.offsets[q]:w.sls.offsets[q + 1]]
        worst = max(worst, relf(T, O.procrustes(w.X[:, sl], w.Y[:, sl])))
    assert worst <= 1e-4, worst
    assert plan.stats()["n_fp64"] == 0


def test_tc_layouts_give_identical_results(gpu):
    """The autotuner's layouts (shared memory per CTA, so CTAs per SM and pipeline depth) change
    the schedule, not the arithmetic: the tuned run and every pinned layout agree bit for bit."""
    import torch
    w = W.small_case(seed=13, nv=642, nt=300, lo=60, hi=200)
    plan = Plan.from_workload(w)
    dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).cuda()
    dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).cuda()
    outs = []
    for layout in (None, (110, 110), (53, 200), (72, 110)):
        if layout is not None:
            plan.set_tc_layout(layout)
        vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
        plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, True, L.SOLVER_TC, L.OUT_CSR)
        torch.cuda.synchronize()
        outs.append(vals.cpu().numpy())
        lay = plan.tc_layout()
        assert lay["tuned"]
        if layout is None:  # the first run tuned both classes (this case has tiles of both)
            assert all(v > 0 for v in lay["candidates_ms"]["le128_cols"].values())
            assert lay["candidates_ms"]["129_256_cols"]["110"] > 0
        else:
            assert tuple(lay["smem_kb"]) == layout
    for o in outs[1:]:
        assert o.tobytes() == outs[0].tobytes()
    with pytest.raises(RuntimeError):
        plan.set_tc_layout((64, 110))


def test_tc_graph_replay_matches_direct_launches(gpu, hlib):
    """The iteration loop captured as a CUDA graph (the default) and replayed gives the same bits as
    launching it kernel by kernel, on the first (capturing) call and on replays."""
    import torch
    w = W.small_case(seed=17, nv=642, nt=200, lo=40, hi=150)
    plan = Plan.from_workload(w)
    dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).cuda()
    dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).cuda()

    def run():
        vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
        plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, True, L.SOLVER_TC, L.OUT_CSC)
        torch.cuda.synchronize()
        return vals.cpu().numpy().tobytes()

    try:
        hlib.ha_b200_set_graphs(False)
        direct = run()
        hlib.ha_b200_set_graphs(True)
        n0 = hlib.ha_b200_launch_count()
        captured = run()
        replayed = run()
        assert hlib.ha_b200_launch_count() > n0
    finally:
        hlib.ha_b200_set_graphs(True)
    assert captured == direct and replayed == direct


_PIPELINE_SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from hyperalignment_b200 import _lib as L
lib = L.lib()
assert lib.ha_b200_init() == 0
out = {}
for n in (16, 100, 200, 272, 512):
    rng = np.random.default_rng(n)
    X = (rng.standard_normal((n, n)) / np.sqrt(n)).astype(np.float32)
    M = (rng.standard_normal((n, n)) / np.sqrt(n)).astype(np.float32)
    for which, b in ((0, None), (1, M)):
        o = np.zeros((n, n), dtype=np.float32)
        fp = L.c_float_p
        rc = lib.ha_b200_tc_selftest(which, n, 0, X.ctypes.data_as(fp), None if b is None else b.ctypes.data_as(fp),
                                     o.ctypes.data_as(fp))
        assert rc == 0
        out[f"{which}_{n}"] = o
np.savez(sys.argv[2], **out)
"""


def test_bulk_and_thread_pipelines_bitwise_equal(gpu, tmp_path):
    """The iteration's products staged by bulk copies (HA_B200_TC_BULK bits), by per-thread loads, or
    by the persistent tile kernel (HA_B200_TC_ITER_FROM=0) feed the same MMAs with the same bytes, so
    every setting gives identical bits."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for mask in ("0", "1", "3", "iter"):
        path = tmp_path / f"m{mask}.npz"
        env = dict(os.environ, HA_B200_TC_ITER_FROM="0") if mask == "iter" else dict(os.environ, HA_B200_TC_BULK=mask)
        subprocess.run([sys.executable, "-c", _PIPELINE_SCRIPT, root, str(path)], env=env, check=True, timeout=300)
        res[mask] = np.load(path)
    for k in res["0"].files:
        assert res["1"][k].tobytes() == res["0"][k].tobytes(), k
        assert res["3"][k].tobytes() == res["0"][k].tobytes(), k
        assert res["iter"][k].tobytes() == res["0"][k].tobytes(), k


_SOLVE_SCRIPT = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import torch
from hyperalignment_b200 import _lib as L
from hyperalignment_b200 import workloads as W
from hyperalignment_b200.plan import Plan
assert L.lib().ha_b200_init() == 0
w = W.rank_deficient_pair(3, nv=642, nt=200)
plan = Plan.from_workload(w)
dX = torch.from_numpy(np.asfortranarray(w.X).ravel(order="F")).cuda()
dY = torch.from_numpy(np.asfortranarray(w.Y).ravel(order="F")).cuda()
vals = torch.zeros(plan.nnz, dtype=torch.float64, device="cuda")
for _ in range(2):
    vals.zero_()
    plan.procrustes_device(dX.data_ptr(), dY.data_ptr(), vals.data_ptr(), True, True, L.SOLVER_TC, L.OUT_CSR)
torch.cuda.synchronize()
np.save(sys.argv[2], vals.cpu().numpy())
"""


def test_iteration_kernels_switch_point_bitwise(gpu, tmp_path):
    """The whole tensor-core solve gives identical bits whichever iteration the persistent kernel
    takes over from (HA_B200_TC_ITER_FROM: always, from iteration 5, never)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for v in ("0", "5", "1000"):
        path = tmp_path / f"f{v}.npy"
        env = dict(os.environ, HA_B200_TC_ITER_FROM=v)
        subprocess.run([sys.executable, "-c", _SOLVE_SCRIPT, root, str(path)], env=env, check=True, timeout=600)
        out[v] = np.load(path)
    assert out["0"].tobytes() == out["1000"].tobytes()
    assert out["5"].tobytes() == out["1000"].tobytes()
