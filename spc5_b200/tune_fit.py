"""Calibration of the autotuner's B200 cost model (csrc/tune.cu).

The model predicts the time of one SpMV through a converted handle's default
kernel choice for rows-per-block r and value type, from numbers the
autotuner gets from the device block counter without converting:

    t_us(r) = t0 + nnz * g(a),   a = nnz / blocks_r (values per block),
    g(a)    = d0 + d1 / a + d2 / a^2   (microseconds per value),

one set of coefficients per value type, r and regime: the row kernel (every
block-row fits its staging buffers: stencils, banded, Poisson) or the
length-sorted plan (some block-row does not: power-law and other irregular
matrices).  d1 / a is the per-block cost spread over the block's values, so
like the reference's SPC5_find_best (src/spc5.hpp:1151-1223) the speed is
keyed by the average number of values per block; the coefficients are
measured on a B200 with this project's kernels, for r = 1, 2, 4 and 8.

    python -m spc5_b200.tune_fit measure > calib.jsonl   # on a B200
    python -m spc5_b200.tune_fit fit calib.jsonl          # prints the C table
    python -m spc5_b200.tune_fit measure_plan > plan.jsonl           # plan regime only
    python -m spc5_b200.tune_fit refit_plan plan.jsonl spc5_b200/csrc/tune.cu

``fit`` prints the table pasted into csrc/tune.cu (kModel) and the fraction of
calibration matrices whose modelled pick is within 10% of the best measured r
(or within 3 us: the timing noise of a launch-bound SpMV).
"""
from __future__ import annotations

import json
import sys

import numpy as np

from . import matrices as M

RS = (1, 2, 4, 8)


def calibration_set():
    """Matrices of the shapes this project serves, spanning 1 to ~60 values
    per block: banded (the batched workload's generator and denser bands),
    27-point stencils, 5-point Poisson, power-law, random."""
    rng = np.random.default_rng(3)
    out = []
    for i in range(24):
        n = int(round(np.exp(rng.uniform(np.log(2e3), np.log(2e5)))))
        bw = int(rng.integers(5, 201))
        out.append(M.banded(n, bw, 0.1, seed=3 * 100003 + i))
    for i in range(24):  # the batched workload's shapes at the sizes where r matters
        n = int(round(np.exp(rng.uniform(np.log(3e4), np.log(4e5)))))
        bw = int(rng.integers(5, 201))
        out.append(M.banded(n, bw, float(rng.choice([0.05, 0.1, 0.2])), seed=5 * 100003 + i))
    for bw, d in ((4, 1.0), (8, 1.0), (16, 0.5), (64, 0.3), (32, 0.8)):
        out.append(M.banded(50_000, bw, d, seed=bw))
    out += [M.stencil27(g) for g in (30, 60, 100)]
    out += [M.poisson2d(g) for g in (128, 256, 512)]
    return out + plan_calibration_set()


def plan_calibration_set():
    """The matrices of the calibration set whose block-rows do not all fit
    the row kernel (the sorted-plan regime): power-law and random."""
    out = [M.powerlaw(n, seed=40 + k) for k, n in enumerate((100_000, 200_000, 300_000, 500_000, 1_000_000,
                                                             2_000_000))]
    for n, per_row, seed in ((200_000, 20, 5), (100_000, 50, 6)):
        g = np.random.default_rng(seed)
        rows = np.repeat(np.arange(n), per_row)
        cols = g.integers(0, n, size=n * per_row)
        out.append(M.from_coo(n, n, rows, cols, g.uniform(-1, 1, size=n * per_row), name=f"random_{n}",
                              sum_duplicates=True))
    return out


def measure(reps: int = 10, warmup: int = 3, mats=None) -> None:
    import torch

    import spc5_b200 as S
    torch.cuda.set_device(0)
    for idx, csr in enumerate(calibration_set() if mats is None else mats):
        for vt in (S.F64, S.F32, S.F32_V8):
            for r in RS:
                dt = np.float64 if vt == S.F64 else np.float32
                m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols,
                                 value_type=S.F32_V8 if vt == S.F32_V8 else None)
                S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
                x = torch.from_numpy(M.x_vector(csr.ncols, 1, dt)).cuda()
                y = torch.zeros(csr.nrows, dtype=torch.float64 if vt != S.F32 else torch.float32, device="cuda")
                f = S.SPC5_Spmv if vt != S.F32_V8 else S.SPC5_Spmv_mixed
                for _ in range(warmup):
                    f(m, x, y)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(reps):
                    f(m, x, y)
                b.record()
                torch.cuda.synchronize()
                print(json.dumps({"idx": idx, "name": csr.name, "vt": vt, "r": r, "nrows": csr.nrows,
                                  "nnz": csr.nnz, "blocks": m.numberOfBlocks,
                                  "plan": int(m.kernel == S.KERNEL_SORTED),
                                  "us": a.elapsed_time(b) * 1e3 / reps}), flush=True)
                del m


def _feats(p):
    a = p["nnz"] / max(1, p["blocks"])
    n = float(p["nnz"])
    return [1.0, n, n / a, n / (a * a)]


def _regime(p):
    """0: row kernel, 1: length-sorted plan (recorded by ``measure``)."""
    return int(p["plan"])


def refit_plan(path: str, table: str) -> None:
    """Refits the sorted-plan rows of the table in ``table`` (a tune.cu) from
    the timings in ``path`` (``measure_plan``), keeping each row's t0: one
    cost per value per value type and r, as ``fit`` does."""
    import re
    src = open(table).read()
    start = src.index("constexpr double kModel")
    body = src[start:src.index("};", start)]
    K = np.array([float(x) for x in re.findall(r"-?\d\.\d+e[+-]\d+", body)]).reshape(3, 4, 2, 4)
    rows = [json.loads(l) for l in open(path) if l.strip()]
    for vt in (0, 1, 2):
        for ri, r in enumerate(RS):
            pts = [p for p in rows if p["vt"] == vt and p["r"] == r and p["plan"] == 1]
            if not pts:
                continue
            t0 = K[vt, ri, 0, 0]
            nnz = np.array([float(p["nnz"]) for p in pts])
            us = np.array([p["us"] for p in pts])
            d0 = float(np.sum((us - t0) / us * nnz / us) / np.sum((nnz / us) ** 2))
            print(f"// value type {vt}, r = {r}: sorted-plan {{t0, d0}} = {{{t0:.6e}, {d0:.6e}}}")


def fit(path: str) -> None:
    rows = [json.loads(l) for l in open(path) if l.strip()]
    for p in rows:
        p["reg"] = _regime(p)
    table = {}
    for vt in (0, 1, 2):
        for r in RS:
            # the row-kernel regime: all four coefficients
            pts = [p for p in rows if p["vt"] == vt and p["r"] == r and p["nnz"] > 0 and p["reg"] == 0]
            f = np.array([_feats(p) for p in pts])
            us = np.array([p["us"] for p in pts])
            w = 1.0 / us  # relative error
            coef, *_ = np.linalg.lstsq(f * w[:, None], us * w, rcond=None)
            table[(vt, r, 0)] = coef
            # the sorted-plan regime has few calibration matrices (their
            # blocks all hold about 2 values): the same t0 and one cost per
            # value (d1 = d2 = 0)
            pts = [p for p in rows if p["vt"] == vt and p["r"] == r and p["nnz"] > 0 and p["reg"] == 1]
            if pts:
                nnz = np.array([float(p["nnz"]) for p in pts])
                us = np.array([p["us"] for p in pts])
                d0 = float(np.sum((us - coef[0]) / us * nnz / us) / np.sum((nnz / us) ** 2))
                table[(vt, r, 1)] = np.array([coef[0], d0, 0.0, 0.0])
            else:
                table[(vt, r, 1)] = coef
    print("// value type (F64, F32, F32_V8) x r (1, 2, 4, 8) x regime (row kernel, sorted plan):")
    print("// t0 [us], d0, d1, d2 [us per value]; t_us = t0 + nnz (d0 + d1 / a + d2 / a^2)")
    print("constexpr double kModel[3][4][2][4] = {")
    for vt in (0, 1, 2):
        print("    {")
        for r in RS:
            rows_s = ", ".join("{" + ", ".join(f"{v:.6e}" for v in table[(vt, r, rg)]) + "}" for rg in (0, 1))
            print(f"        {{{rows_s}}},")
        print("    },")
    print("};")
    by = {}
    for p in rows:
        by.setdefault((p["idx"], p["vt"]), {})[p["r"]] = p
    ok = 0
    for key, d in by.items():
        def model(q):
            return max(float(np.dot(table[(key[1], q["r"], q["reg"])], _feats(q))), 1.0)

        pick = min(d.values(), key=model)
        best = min(q["us"] for q in d.values())
        ok += pick["us"] <= max(1.10 * best, best + 3.0)
    print(f"// modelled pick within 10% (or 3 us) of the best measured r: {ok}/{len(by)}")


if __name__ == "__main__":
    if len(sys.argv) >= 2 and sys.argv[1] == "measure":
        measure()
    elif len(sys.argv) >= 2 and sys.argv[1] == "measure_plan":
        measure(mats=plan_calibration_set())
    elif len(sys.argv) >= 4 and sys.argv[1] == "refit_plan":
        refit_plan(sys.argv[2], sys.argv[3])
    elif len(sys.argv) >= 3 and sys.argv[1] == "fit":
        fit(sys.argv[2])
    else:
        print(__doc__)
