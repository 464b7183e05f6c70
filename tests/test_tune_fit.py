"""The autotuner's calibration scripts on the CPU (no timings are taken).

``fit`` turns timings into the cost-model table of csrc/tune.cu and
``refit_plan`` refits its sorted-plan rows; both are checked here on
synthetic timings made from known coefficients, which they must recover.
"""
import json
import os
import re

import numpy as np

from spc5_b200 import tune_fit as T

TUNE_CU = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "spc5_b200", "csrc", "tune.cu")


def _table():
    src = open(TUNE_CU).read()
    start = src.index("constexpr double kModel")
    body = src[start:src.index("};", start)]
    return np.array([float(x) for x in re.findall(r"-?\d\.\d+e[+-]\d+", body)]).reshape(3, 4, 2, 4)


def test_refit_plan_recovers_the_per_value_cost(tmp_path, capsys):
    K = _table()
    d0 = {(vt, r): 1e-6 * (1 + vt + ri) for vt in range(3) for ri, r in enumerate(T.RS)}
    rows = []
    for vt in range(3):
        for ri, r in enumerate(T.RS):
            for nnz in (1e6, 3e6, 1e7, 3e7):
                rows.append({"vt": vt, "r": r, "plan": 1, "nnz": nnz, "blocks": nnz / 2,
                             "us": K[vt, ri, 0, 0] + nnz * d0[(vt, r)]})
            rows.append({"vt": vt, "r": r, "plan": 0, "nnz": 1e6, "blocks": 5e5, "us": 1e9})  # ignored
    path = tmp_path / "plan.jsonl"
    path.write_text("\n".join(json.dumps(p) for p in rows))
    T.refit_plan(str(path), TUNE_CU)
    out = capsys.readouterr().out
    got = {(int(m.group(1)), int(m.group(2))): float(m.group(4))
           for m in re.finditer(r"value type (\d), r = (\d): sorted-plan \{t0, d0\} = \{([^,]+), ([^}]+)\}", out)}
    assert len(got) == 12
    for key, want in d0.items():
        assert abs(got[key] - want) <= 1e-3 * want, (key, got[key], want)


def test_fit_recovers_a_row_kernel_model(tmp_path, capsys):
    # t = t0 + nnz (d0 + d1 / a + d2 / a^2) for every (value type, r); no
    # plan-regime points: the plan rows fall back to the row-kernel fit
    true = np.array([10.0, 2e-6, 8e-6, 1e-5])
    rows, idx = [], 0
    for a in (1.5, 2.0, 3.0, 5.0, 8.0, 12.0):
        for nnz in (1e5, 1e6, 1e7):
            for vt in range(3):
                for r in T.RS:
                    f = np.array([1.0, nnz, nnz / a, nnz / (a * a)])
                    rows.append({"idx": idx, "vt": vt, "r": r, "plan": 0, "nnz": nnz, "blocks": nnz / a,
                                 "us": float(f @ true)})
            idx += 1
    path = tmp_path / "calib.jsonl"
    path.write_text("\n".join(json.dumps(p) for p in rows))
    T.fit(str(path))
    out = capsys.readouterr().out
    nums = [float(x) for x in re.findall(r"-?\d\.\d+e[+-]\d+", out.split("constexpr double kModel")[1])]
    K = np.array(nums[:96]).reshape(3, 4, 2, 4)
    assert np.allclose(K[:, :, 0, :], true, rtol=1e-4, atol=1e-9)
