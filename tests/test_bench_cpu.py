"""The CPU-side legs of bench.py: the reference arm and the CPU baseline
helper run on a small matrix and report well-formed numbers (no GPU)."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not (oracle.ref_available() and oracle.cpu_has_avx512()),
                               reason="compiled reference or AVX-512 host not available")


@needs_ref
def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--size", "20000", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "GB/s"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


@needs_ref
def test_cpu_baseline_runs_the_reference_arm_in_a_subprocess():
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    args = argparse.Namespace(workload="powerlaw", size=20000)
    cpu = bench.cpu_baseline_subprocess(args, steps=2)
    assert cpu is not None
    assert cpu["kind"] == "reference" and cpu["value"] > 0 and cpu["cores"] >= 1
    assert "separate process" in cpu["sample"]


@needs_ref
def test_reference_arm_config_matches_the_gpu_arm():
    """The reference arm's config dict is built by the same helper as the GPU
    arm's, from the same conversion block counts."""
    sys.path.insert(0, ROOT)
    import bench
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--size", "20000", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    d = json.loads(out.stdout.strip().splitlines()[-1])
    csr = bench.build_workload("powerlaw", 20000)
    blocks = {r: oracle.block_count(r, csr.rowptr, csr.colidx) for r in bench.FORMATS}
    want = bench.spmv_config("powerlaw", csr, blocks, 1, bench.L2_NOTE_LARGE if
                             min(bench.spmv_bytes(csr.nnz, blocks[r], r, csr.nrows, csr.ncols)
                                 for r in bench.FORMATS) >= bench.L2_BYTES else bench.L2_NOTE_FLUSH)
    assert d["config"] == json.loads(json.dumps(want))
