"""bench.py's reference arm on the CPU: the compiled reference (oracle/_ref) timed through the
bench contract, one JSON line from rank 0 only, also when launched as two ranks."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ref_built():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libhyperalignment.so"))


def _lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


@pytest.mark.skipif(not _ref_built(), reason="compiled reference not built (make -C oracle)")
def test_reference_arm_one_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--nv", "642", "--ref-seconds", "0.5"], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "searchlights/s"
    assert d["higher_is_better"] is True and d["cpu_baseline"]["kind"] == "reference"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


@pytest.mark.skipif(not _ref_built(), reason="compiled reference not built (make -C oracle)")
def test_reference_arm_two_ranks_rank0_only():
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", "29517", "bench.py", "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0", "--nv", "642", "--ref-seconds", "0.5"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2
