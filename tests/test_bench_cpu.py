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
def test_cpu_baseline_helper():
    sys.path.insert(0, ROOT)
    import bench
    from spc5_b200 import matrices as M
    res = bench.cpu_baseline(M.poisson2d(64), budget_s=0.2, formats=(1, 4))
    assert res is not None
    gbs, threads, steps, secs = res
    assert gbs > 0 and threads >= 1 and steps >= 1 and secs > 0
