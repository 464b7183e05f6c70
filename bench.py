#!/usr/bin/env python3
"""Benchmark of the beta(r,VS) SpMV hot path on B200 -- one JSON line.

Workload (default): FP64 SpMV across all formats beta(1,8), beta(2,8),
beta(4,8), beta(8,8) on the seeded power-law matrix (N = 4,000,000, row
lengths min(2000, Zipf(1.8) + 3), 70% of each row in diagonal-centred runs,
values U[-1,1], seed 1; ~63.4M nnz, int32 indices).  One step = one
y += A x per format (4 SpMV launches), inputs resident in HBM.

* ``value``   -- algorithmic GB/s of the whole step (bytes of values,
  headers, block-row pointer, x once and y read+write, per SpMV), summed
  over ranks, divided by the max-over-ranks device time.
* ``e2e``     -- the same bytes per step over the time of the public call
  sequence with HOST buffers: pinned x and y copied in, the 4 SpMVs, y
  copied back, every step.
* ``roofline``-- the SpMV kernel: algorithmic bytes per launch / mean
  CUDA-event launch time, against the measured HBM copy bandwidth.
* ``mixed``   -- the same matrix with float values in the 8-column layout
  (uint8 masks), FP32 x and FP64 accumulation: GB/s, SpMV/s ratio to FP64
  and the error against an FP64 CSR product (per row relative to
  sum_j |a_ij x_j|, and normwise); ``mixed.f32_layout`` is the same for the
  reference's float layout beta(r,16).
* ``cpu_baseline`` -- the reference's own AVX-512 OpenMP SpMV
  (SPC5_Spmv_omp, src/spc5.hpp compiled by oracle/Makefile) on this host.

``--impl reference`` runs only the reference CPU path with all host
threads and prints its line.  Multi-GPU (torchrun): every rank runs its own
copy of the workload (weak scaling); only barrier and max-reduction of the
timings cross ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from spc5_b200 import matrices as M  # noqa: E402

METRIC = "SpMV GB/s (algorithmic bytes, FP64, all beta(r,8) formats)"
UNIT = "GB/s"
FORMATS = (1, 2, 4, 8)


def spmv_bytes(nnz, nblocks, r, nrows, ncols, value_bytes=8, mask_bytes=1, x_bytes=8, y_bytes=8):
    """Algorithmic bytes of one y += A x in beta(r,VS):
    nnz*sv + blocks*(4 + r*m) + 4*(ceil(N/r)+1) + ncols*sx + 2*N*sy."""
    nbr = (nrows + r - 1) // r
    return (nnz * value_bytes + nblocks * (4 + r * mask_bytes) + 4 * (nbr + 1) + ncols * x_bytes
            + 2 * nrows * y_bytes)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def build_workload(name, size=None):
    if name == "powerlaw":
        return M.powerlaw(size or 4_000_000)
    if name == "stencil27":
        return M.stencil27(size or 160)
    if name == "poisson":
        return M.poisson2d(512)
    raise ValueError(name)


def workload_desc(name, csr):
    return {"powerlaw": f"power-law N={csr.nrows:,} Zipf(1.8)+3 clipped to 2000, 70% runs U[1,16] near "
                        "diagonal (sigma N/100), U[-1,1] values, seed 1",
            "stencil27": f"27-point stencil {round(csr.nrows ** (1 / 3))}^3, diag 26, neighbours "
                         "-1+U[-1e-3,1e-3], seed 2",
            "poisson": "5-point Poisson 512^2, diag 4, off -1"}[name] + f"; nnz={csr.nnz}"


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = None
        self.thread = None
        self.rows = []
        self.stop = False

    # NVML clocks-event reason bits (nvml.h): read-only queries, nothing is set
    _REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
                    "hw_thermal_slowdown": 0x40}

    def _poll_nvml(self, h, nv):
        try:
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        except Exception:
            mx = None
        self._mx = mx
        while not self.stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                try:
                    bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                except Exception:
                    bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((sm, mx, bits))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            import threading
            self.thread = threading.Thread(target=self._poll_nvml, args=(h, nv), daemon=True)
            self.thread.start()
            self._h, self._nv = h, nv
            return self
        except Exception:
            self.thread = None
        try:
            self.out = open(f"/tmp/spc5_clocks_{os.getpid()}.csv", "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def sample_now(self):
        """One synchronous sample (the polling thread may be starved in a short region)."""
        if self.thread is None:
            return
        nv, h = self._nv, self._h
        try:
            try:
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            self.rows.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                              nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM), bits))
        except Exception:
            pass

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop = True
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.out:
            self.out.close()

    def summary(self):
        if self.thread is not None:
            if not self.rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            sm = [r[0] for r in self.rows]
            mx = [r[1] for r in self.rows if r[1]]
            reasons = sorted({n for r in self.rows for n, b in self._REASON_BITS.items() if r[2] & b})
            load = [v for v in sm if mx and v > 0.3 * max(mx)] or sm
            return {"sm_mhz": statistics.median(load), "sm_max_mhz": max(mx) if mx else None,
                    "reasons": reasons, "samples": len(self.rows), "source": "nvml, 2 ms"}
        path = f"/tmp/spc5_clocks_{os.getpid()}.csv"
        if not os.path.exists(path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        rows = []
        with open(path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        load = [s for s in sm if mx and s > 0.3 * max(mx)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's OpenMP path
# ---------------------------------------------------------------------------

def cpu_baseline_subprocess(args, steps=16):
    """The reference's own AVX-512 OpenMP SpMV on this host, run as the
    reference arm in a separate process (``bench.py --impl reference``) with
    all host threads and nothing else running: {value, unit, cores, kind,
    sample}, or None when the reference is not available here."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--workload", args.workload,
           "--steps", str(steps), "--warmup", "1", "--formats", ",".join(str(r) for r in FORMATS),
           "--gpus", "1"]
    if args.size is not None:
        cmd += ["--size", str(args.size)]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        res = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
        line = json.loads(res.stdout.strip().splitlines()[-1])
    except Exception:
        return None
    if "unavailable" in line:
        return None
    cpu = dict(line["cpu_baseline"])
    cpu["sample"] += "; separate process (bench.py --impl reference), before the GPU legs"
    return cpu


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libspc5ref.so was not built"}))
        return 0
    if not oracle.cpu_has_avx512():
        print(json.dumps({"impl": "reference", "unavailable": "host CPU has no AVX-512 (reference build "
                                                               "uses USE_AVX512 kernels)"}))
        return 0
    csr = build_workload(args.workload, args.size)
    threads = oracle.ref().ref_max_threads()
    xp = oracle.x_padded(M.x_vector(csr.ncols, 0))
    mats, step_bytes, blocks, bytes_of = [], 0, {}, []
    for r in FORMATS:
        m = oracle.RefMatrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
        nb = m.convert(r)
        m.split(threads)
        mats.append(m)
        blocks[r] = nb
        bytes_of.append(spmv_bytes(csr.nnz, nb, r, csr.nrows, csr.ncols))
        step_bytes += bytes_of[-1]
    y = np.zeros(csr.nrows + 8)
    for _ in range(args.warmup):
        for m in mats:
            m.time_spmv_omp(xp, y, 1)
    secs = 0.0
    for _ in range(args.steps):
        for m in mats:
            secs += m.time_spmv_omp(xp, y, 1)
    value = step_bytes * args.steps / secs / 1e9
    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(secs / args.steps * 1e3, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": spmv_config(args.workload, csr, blocks, args.gpus,
                                  L2_NOTE_FLUSH if min(bytes_of) < L2_BYTES else L2_NOTE_LARGE),
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{args.steps} steps x {len(FORMATS)} SPC5_Spmv_omp calls (r={FORMATS}) on the "
                                       f"full matrix, OMP threads={threads}"},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU path
# ---------------------------------------------------------------------------

def fp64_csr_reference(csr, x):
    """FP64 CSR product y = A x and sum_j |a_ij x_j| per row, on the device
    (cuSPARSE through torch.sparse): the yardstick of the mixed-precision
    error, independent of the beta kernels."""
    import torch
    rp = torch.from_numpy(csr.rowptr.astype(np.int64)).cuda()
    ci = torch.from_numpy(csr.colidx.astype(np.int64)).cuda()
    va = torch.from_numpy(csr.values).cuda()
    a = torch.sparse_csr_tensor(rp, ci, va, (csr.nrows, csr.ncols))
    y = (a @ x.unsqueeze(1)).squeeze(1)
    a_abs = torch.sparse_csr_tensor(rp, ci, va.abs(), (csr.nrows, csr.ncols))
    absrow = (a_abs @ x.abs().unsqueeze(1)).squeeze(1)
    del a, a_abs, rp, ci, va
    return y, absrow


def mixed_legs(csr, mats, x, per_r_ms, args, stream, select_kernel):
    """Mixed precision on the bench matrix for every format: GB/s, SpMV/s
    relative to the FP64 path, and the error against an FP64 CSR product.
    ``mixed`` is the 8-column layout (F32_V8: float values, uint8 masks);
    ``f32_layout`` the reference's float layout beta(r,16)."""
    import torch
    import spc5_b200 as S
    y64, absrow = fp64_csr_reference(csr, x)
    x32 = x.float()
    out = {}
    for name, vt, (sv, mb) in (("v8", S.F32_V8, (4, 1)), ("f32_layout", S.F32, (4, 2))):
        ms_total, fp64_total, nbytes, comp, normw = 0.0, 0.0, 0, 0.0, 0.0
        for r, _m64 in mats:
            mm = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols, dtype=np.float32, value_type=vt)
            S.CSR_to_SPC5(mm, S.FORMAT_OF_R[r])
            select_kernel(mm, args.kernel)
            ym = torch.zeros(csr.nrows, dtype=torch.float64, device="cuda")
            S.SPC5_Spmv_mixed(mm, x32, ym)
            torch.cuda.synchronize()
            d = (ym - y64).abs()
            comp = max(comp, (d / absrow.clamp_min(1e-300)).max().item())
            normw = max(normw, (d.max() / y64.abs().max()).item())
            for _ in range(args.warmup):
                S.SPC5_Spmv_mixed(mm, x32, ym)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                S.SPC5_Spmv_mixed(mm, x32, ym)
            b.record(stream)
            torch.cuda.synchronize()
            ms_total += a.elapsed_time(b) / args.steps
            fp64_total += per_r_ms[r]
            nbytes += spmv_bytes(csr.nnz, mm.numberOfBlocks, r, csr.nrows, csr.ncols, sv, mb, 4, 8)
            del mm, ym
        out[name] = {"gbs": round(nbytes / (ms_total * 1e-3) / 1e9, 2),
                     "spmv_per_s_ratio_vs_fp64": round(fp64_total / ms_total, 3),
                     "max_componentwise_rel_err_vs_fp64_csr": comp,
                     "normwise_rel_err_vs_fp64_csr": normw}
    del y64, absrow
    res = dict(out["v8"])
    res["layout"] = "float values in the 8-column layout (uint8 masks), FP32 x, FP64 accumulation and y"
    res["error_reference"] = "FP64 CSR product of the unrounded matrix and x (cuSPARSE via torch); componentwise = max_i |dy_i| / sum_j |a_ij x_j|"
    res["f32_layout"] = out["f32_layout"]
    return res


def spmv_config(workload, csr, blocks, nranks, l2_note):
    """The ``config`` dict of an SpMV line, identical in both arms."""
    return {"workload": workload, "desc": workload_desc(workload, csr), "formats": list(FORMATS),
            "nrows": csr.nrows, "nnz": csr.nnz, "blocks": {str(r): int(blocks[r]) for r in FORMATS},
            "l2": l2_note, "parallelism": f"replica per GPU x{nranks}"}


L2_NOTE_LARGE = "inputs larger than L2 (every matrix > 126 MB, read in turn)"
L2_NOTE_FLUSH = "L2 flushed (256 MB write) before every SpMV; value from the SpMVs' own CUDA events"


def dropin_leg(mats, csr, x, steps, warmup, stream):
    """The reference-named void symbols core_SPC5_{r}rVc_Spmv_double over
    device copies of the converted arrays (no handle): per call the library
    derives the block-row offsets and splits on the device and runs the row
    kernel when every block-row fits it, else the group kernel."""
    import torch

    import spc5_b200 as S
    per, total_bytes, total_ms = {}, 0, 0.0
    y = torch.zeros(csr.nrows, dtype=torch.float64, device=x.device)
    for r, m in mats:
        b, h, v = m.arrays()
        bd, hd, vd = (torch.from_numpy(a).to(x.device) for a in (b, h, v))
        for _ in range(warmup):
            S.core_spmv_void(r, csr.nrows, bd, hd, vd, x, y, stream)
        torch.cuda.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            S.core_spmv_void(r, csr.nrows, bd, hd, vd, x, y, stream)
        e.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(e) / steps
        nbytes = spmv_bytes(csr.nnz, m.numberOfBlocks, r, csr.nrows, csr.ncols)
        per[str(r)] = round(nbytes / (ms * 1e-3) / 1e9, 2)
        total_bytes += nbytes
        total_ms += ms
        del bd, hd, vd
    return {"value": round(total_bytes / (total_ms * 1e-3) / 1e9, 2), "unit": UNIT, "per_format_gbs": per,
            "call": "core_SPC5_{r}rVc_Spmv_double (void, reference argument list, device pointers)"}


def spmv_leg(csr, args, dev, world, barrier, max_over_ranks, steps, warmup, e2e=True, mixed=True,
             dropin=False):
    """One SpMV workload on this GPU: every format converted on the device,
    then the device-timed steps (one y += A x per format), per-format GB/s,
    the launch-level roofline, the end-to-end rate through the public API with
    host buffers, and the mixed-precision legs."""
    import torch

    import spc5_b200 as S
    stream = torch.cuda.current_stream()
    mats, bytes_of = [], {}
    for r in FORMATS:
        m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values, csr.ncols)
        S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
        select_kernel(m, args.kernel)
        mats.append((r, m))
        bytes_of[r] = spmv_bytes(csr.nnz, m.numberOfBlocks, r, csr.nrows, csr.ncols)
    step_bytes = sum(bytes_of.values())
    x = torch.from_numpy(M.x_vector(csr.ncols, 0)).to(dev)
    y = torch.zeros(csr.nrows, dtype=torch.float64, device=dev)
    # a matrix smaller than L2 would be read from L2 in the next step: flush
    # L2 (a 256 MB write) before every SpMV and time the SpMVs alone
    flush = None
    if min(bytes_of.values()) < L2_BYTES:
        flush = torch.empty(64 * 2**20, dtype=torch.float32, device=dev)

    def step(events=None, cold=True):
        for i, (r, m) in enumerate(mats):
            if flush is not None and cold:
                flush.zero_()
            if events is not None:
                events[i][0].record(stream)
            S.SPC5_Spmv(m, x, y)
            if events is not None:
                events[i][1].record(stream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()

    # ---- device-timed region (inputs resident, larger than L2) ----
    launch_ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in mats] for _ in range(steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        barrier()
        torch.cuda.synchronize()
        t_start.record(stream)
        for k in range(steps):
            step(launch_ev[k])
        t_end.record(stream)
        clk.sample_now()  # the queued steps are still running
        torch.cuda.synchronize()
        barrier()
    clocks = clk.summary()
    ms_local = t_start.elapsed_time(t_end)
    per_r_ms = {r: statistics.mean(launch_ev[k][i][0].elapsed_time(launch_ev[k][i][1]) for k in range(steps))
                for i, (r, _) in enumerate(mats)}
    kernel_ms = sum(per_r_ms.values())
    if flush is not None:
        ms_local = kernel_ms * steps  # the SpMVs without the flushes between them
    ms = max_over_ranks(ms_local)
    value = step_bytes * steps * world / (ms * 1e-3) / 1e9
    warm = None
    if flush is not None:
        # the same steps back to back without flushes: the matrices stay in L2
        barrier()
        torch.cuda.synchronize()
        w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0.record(stream)
        for _ in range(steps):
            step(cold=False)
        w1.record(stream)
        torch.cuda.synchronize()
        wms = max_over_ranks(w0.elapsed_time(w1))
        warm = {"value": round(step_bytes * steps * world / (wms * 1e-3) / 1e9, 2), "unit": UNIT,
                "note": "no L2 flush between SpMVs: the matrices stay in L2"}
    achieved = step_bytes / (kernel_ms * 1e-3) / 1e9
    peak, peak_kind = load_peaks()
    out = {"value": value, "ms": ms, "step_bytes": step_bytes, "mats": mats, "x": x, "y": y,
           "blocks": {r: m.numberOfBlocks for r, m in mats}, "flush": flush is not None,
           "memory": {"device_gb": {str(r): round(m.info().device_bytes / 1e9, 3) for r, m in mats},
                      "beta_gb": {str(r): round((m.info().header_bytes + csr.nnz * 8) / 1e9, 3) for r, m in mats},
                      "note": "handle footprint on the device against its beta(r,8) headers and values"},
           "per_format_gbs": {str(r): round(bytes_of[r] / (per_r_ms[r] * 1e-3) / 1e9, 2) for r in FORMATS},
           "per_r_ms": per_r_ms, "bytes_of": bytes_of, "achieved": achieved, "peak": peak,
           "peak_kind": peak_kind, "clocks": clocks, "warm": warm,
           "gflops": 2 * csr.nnz * len(FORMATS) * steps * world / (ms * 1e-3) / 1e9}

    if e2e:
        # ---- e2e through the public API with host buffers ----
        # Every step copies its own x and y in from pinned host memory, runs
        # the SpMVs and copies its y back.  Steps alternate between two
        # streams with their own device and host buffers, so one step's copies
        # overlap the previous step's kernels (what a caller streaming
        # requests does).
        x_host = torch.from_numpy(M.x_vector(csr.ncols, 0)).pin_memory()
        e2e_streams = [torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)]
        e2e_bufs = [(torch.empty_like(x), torch.empty_like(y),
                     torch.zeros(csr.nrows, dtype=torch.float64).pin_memory(),
                     torch.zeros(csr.nrows, dtype=torch.float64).pin_memory()) for _ in range(2)]

        def e2e_step(k):
            xd, yd, yh_in, yh_out = e2e_bufs[k % 2]
            with torch.cuda.stream(e2e_streams[k % 2]):
                xd.copy_(x_host, non_blocking=True)
                yd.copy_(yh_in, non_blocking=True)
                for r, m in mats:
                    S.SPC5_Spmv(m, xd, yd)
                yh_out.copy_(yd, non_blocking=True)

        for k in range(max(1, warmup)):
            e2e_step(k)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for st in e2e_streams:
            st.wait_event(e0)
        for k in range(steps):
            e2e_step(k)
        for st in e2e_streams:
            stream.wait_stream(st)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1))
        out["e2e"] = {"value": round(step_bytes * steps * world / (e2e_ms * 1e-3) / 1e9, 2), "unit": UNIT,
                      "h2d_bytes_per_step": int(x.numel() * 8 + y.numel() * 8),
                      "d2h_bytes_per_step": int(y.numel() * 8)}

    if dropin:
        out["dropin"] = dropin_leg(mats, csr, x, steps, warmup, stream)

    # ---- mixed precision on the same matrix: float values and x, FP64
    # accumulation and y, in the 8-column layout (F32_V8, the default) and in
    # the reference's float layout (beta(r,16)); the error is stated against an
    # FP64 CSR product of the unrounded matrix and x on the device (cuSPARSE
    # through torch), per row relative to sum_j |a_ij x_j| and normwise
    out["mixed"] = {}
    if mixed:
        a2 = argparse.Namespace(**vars(args))
        a2.steps, a2.warmup = steps, warmup
        out["mixed"] = mixed_legs(csr, mats, x, per_r_ms, a2, stream, select_kernel)
    return out


def run_gpu(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # the CPU baseline first, in its own process, before this process touches
    # the GPU (rank 0 at N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_subprocess(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    csr = build_workload(args.workload, args.size)
    main = spmv_leg(csr, args, dev, world, barrier, max_over_ranks, args.steps, args.warmup,
                    mixed=not args.no_mixed, dropin=(world == 1 and not args.no_extra))
    mats = main["mats"]
    traffic, traffic_src = args.traffic, "ncu (given)" if args.traffic else None
    ratios = TRAFFIC_RATIO.get(args.workload)
    if traffic is None and ratios and args.kernel == "auto" and all(r in ratios for r in FORMATS):
        traffic = int(sum(ratios[r] * main["bytes_of"][r] for r in FORMATS))
        traffic_src = "ncu DRAM bytes per algorithmic byte at a smaller size of the same generator, scaled"
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(main["value"], 2), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(main["ms"] / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": spmv_config(args.workload, csr, main["blocks"], world,
                                  L2_NOTE_FLUSH if main["flush"] else L2_NOTE_LARGE),
            "per_format_gbs": main["per_format_gbs"],
            "gflops": round(main["gflops"], 2),
            "roofline": {"bound": "hbm", "achieved": round(main["achieved"], 2), "peak": main["peak"],
                         "unit": "GB/s", "frac": round(main["achieved"] / main["peak"], 4),
                         "peak_kind": main["peak_kind"], "traffic": traffic, "traffic_source": traffic_src,
                         "kernel": ", ".join(sorted({KERNEL_NAME[m.kernel] for _, m in mats}))},
            "kernels": {str(r): KERNEL_NAME[m.kernel] for r, m in mats},
            "memory": main["memory"],
            "e2e": main["e2e"],
            "gpu_launches": sum(m.spmv_launches for _, m in mats) * args.steps,
            "clocks": main["clocks"],
            "mixed": main["mixed"],
        }
        if "dropin" in main:
            line["dropin"] = main["dropin"]
        if main["warm"] is not None:
            line["warm"] = main["warm"]
    del main, mats
    torch.cuda.empty_cache()
    # ---- the other configurations of the metric, on this GPU (N = 1 only):
    # the 27-point stencil 160^3 (FP64 vs mixed), the 5-point Poisson 512^2
    # (L2-resident: cold and warm) and a short serving run
    if world == 1 and args.workload == "powerlaw" and args.size is None and not args.no_extra:
        extra_steps, extra_warm = max(5, args.steps // 2), 3
        for name, key in (("stencil27", "config3_stencil27_160"), ("poisson", "config1_poisson_512")):
            c2 = build_workload(name)
            leg = spmv_leg(c2, args, dev, world, barrier, max_over_ranks, extra_steps, extra_warm,
                           e2e=False, mixed=(name == "stencil27" and not args.no_mixed),
                           dropin=(name == "stencil27"))
            entry = {"value": round(leg["value"], 2), "unit": UNIT, "steps": extra_steps,
                     "config": spmv_config(name, c2, leg["blocks"], world,
                                           L2_NOTE_FLUSH if leg["flush"] else L2_NOTE_LARGE),
                     "per_format_gbs": leg["per_format_gbs"],
                     "roofline_frac": round(leg["achieved"] / leg["peak"], 4),
                     "kernels": {str(r): KERNEL_NAME[m.kernel] for r, m in leg["mats"]},
                     "clocks": leg["clocks"]}
            if leg["mixed"]:
                entry["mixed"] = leg["mixed"]
            if "dropin" in leg:
                entry["dropin"] = leg["dropin"]
            if leg["warm"] is not None:
                entry["warm"] = leg["warm"]
            line[key] = entry
            line["gpu_launches"] += sum(m.spmv_launches for _, m in leg["mats"]) * extra_steps
            del leg, c2
            torch.cuda.empty_cache()
        line["config5_serving"] = serve_leg(args, rates=(5000.0, 50000.0), seconds=1.0, precisions=(False,))
    if rank == 0:
        line["cpu_baseline"] = cpu
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# sharded: one matrix split across the ranks by block-row ranges, iterated
# ---------------------------------------------------------------------------

def run_sharded(args):
    """--mode sharded: the power-law (or --workload) matrix cut into equal
    block-row ranges, one per rank; a step is, for every format, one
    iteration x <- A x: the NCCL all-gather of the x slices (in place, no
    copy of x) and the local SpMV.  Strong scaling: the matrix is fixed."""
    import torch
    import torch.distributed as dist

    from spc5_b200 import distributed as D
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    csr = build_workload(args.workload, args.size)
    if csr.nrows != csr.ncols:
        raise SystemExit("sharded iteration needs a square matrix")
    shards, local_bytes = [], 0
    for r in FORMATS:
        sh = D.ShardedSpMV(csr, rank, world, r, dev, cuts="equal")
        shards.append((r, sh))
        nb = sh.mat.numberOfBlocks
        local_bytes += spmv_bytes(sh.local.nnz, nb, r, sh.local.nrows, csr.ncols)
    x0 = torch.from_numpy(M.x_vector(csr.ncols, 0)).to(dev)
    xs = {r: x0[sh.r0:sh.r1].clone() for r, sh in shards}
    stream = torch.cuda.current_stream()

    def step(ev=None):
        for i, (r, sh) in enumerate(shards):
            if ev is not None:
                ev[i][0].record(stream)
            xf = sh.gather_x(xs[r])
            if ev is not None:
                ev[i][1].record(stream)
            y = torch.zeros(sh.r1 - sh.r0, dtype=torch.float64, device=dev)
            sh.local_spmv(xf, y)
            # keep the iterate bounded: x <- A x / max|A x| would need a
            # reduction; y is scaled by a constant instead (the bytes and the
            # exchange are the same)
            xs[r] = y.mul_(0.05)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in shards] for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t0.record(stream)
        for k in range(args.steps):
            step(ev[k])
        t1.record(stream)
        clk.sample_now()
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    gather_ms = sum(ev[k][i][0].elapsed_time(ev[k][i][1]) for k in range(args.steps) for i in range(len(shards)))
    vals = torch.tensor([ms, gather_ms, float(local_bytes)], dtype=torch.float64, device=dev)
    per_rank = [vals.clone() for _ in range(world)]
    if world > 1:
        dist.all_gather(per_rank, vals)
    ms_max = max(float(v[0]) for v in per_rank)
    total_bytes = sum(float(v[2]) for v in per_rank)
    line = None
    if rank == 0:
        line = {"metric": METRIC + ", sharded iteration", "value": round(total_bytes * args.steps / (ms_max * 1e-3) / 1e9, 2),
                "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": args.workload, "desc": workload_desc(args.workload, csr),
                           "formats": list(FORMATS), "nrows": csr.nrows, "nnz": csr.nnz,
                           "parallelism": f"block-row shards x{world}, NCCL all-gather of x per iteration"},
                "per_rank": [{"rank": k, "gbs": round(float(v[2]) * args.steps / (float(v[0]) * 1e-3) / 1e9, 2),
                              "allgather_us_per_step": round(float(v[1]) * 1e3 / args.steps, 1)}
                             for k, v in enumerate(per_rank)],
                "clocks": clk.summary(),
                "gpu_launches": sum(sh.mat.spmv_launches for _, sh in shards) * args.steps}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# batched workload: many banded matrices, per-matrix r, k right-hand sides
# ---------------------------------------------------------------------------

def batched_matrices(count=256, seed=3):
    """Banded matrices with N log-uniform in [2e3, 2e5], bandwidth U[5, 200],
    density 0.1 in the band, values U[-1, 1]; k in {1, 4, 8, 16}."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(2e3), np.log(2e5)))))
        bw = int(rng.integers(5, 201))
        k = int(rng.choice([1, 4, 8, 16]))
        out.append((M.banded(n, bw, 0.1, seed=seed * 100003 + i), k))
    return out


def run_batched(args):
    import torch

    import spc5_b200 as S
    torch.cuda.set_device(0)
    work = batched_matrices(args.batch_count)
    lines = []
    for mixed in (False, True):
        dt = np.float32 if mixed else np.float64
        tdt = torch.float32 if mixed else torch.float64
        mats, Xs, Ys, total_bytes, flops, chosen = [], [], [], 0, 0, {}
        for csr, k in work:
            m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols,
                             value_type=S.F32_V8 if mixed else None)
            r = S.autotune(m, S.TUNE_MODEL)["r"]
            S.CSR_to_SPC5(m, S.FORMAT_OF_R[r])
            chosen[r] = chosen.get(r, 0) + 1
            mats.append(m)
            Xs.append(torch.from_numpy(np.random.default_rng(len(Xs)).uniform(-1, 1, (csr.ncols, k))).to(
                "cuda", tdt))
            Ys.append(torch.zeros(csr.nrows, k, dtype=torch.float64 if mixed else tdt, device="cuda"))
            sv, mb, sx = (4, 1, 4) if mixed else (8, 1, 8)
            nbr = (csr.nrows + r - 1) // r
            total_bytes += (csr.nnz * sv + m.numberOfBlocks * (4 + r * mb) + 4 * (nbr + 1) +
                            k * (csr.ncols * sx + 2 * csr.nrows * 8))
            flops += 2 * csr.nnz * k
        batch = S.Batch(mats, Xs, Ys, mixed=mixed)
        nclasses, njobs = batch.info()
        for _ in range(args.warmup):
            batch.launch()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            batch.launch()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.steps
        lines.append({"precision": "mixed" if mixed else "f64", "ms_per_step": round(ms, 4),
                      "gbs": round(total_bytes / (ms * 1e-3) / 1e9, 2),
                      "gflops": round(flops / (ms * 1e-3) / 1e9, 2),
                      "spmv_per_s": round(sum(k for _, k in work) / (ms * 1e-3), 1),
                      "graph_classes": nclasses, "jobs": njobs,
                      "r_chosen": {str(r): c for r, c in sorted(chosen.items())}})
        del batch, mats, Xs, Ys
        torch.cuda.empty_cache()
    peak, peak_kind = load_peaks()
    line = {"metric": "batched SpMM GB/s (algorithmic bytes, one CUDA graph)", "value": lines[0]["gbs"],
            "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": lines[0]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched", "matrices": len(work),
                       "desc": "banded, N log-uniform [2e3,2e5], bandwidth U[5,200], density 0.1, "
                               "k in {1,4,8,16}, seed 3, r per matrix by the autotuner (model)",
                       "nnz": int(sum(c.nnz for c, _ in work))},
            "precisions": lines,
            "roofline": {"bound": "hbm", "achieved": lines[0]["gbs"], "peak": peak, "unit": "GB/s",
                         "frac": round(lines[0]["gbs"] / peak, 4), "peak_kind": peak_kind}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# serving workload: resident pool, Poisson arrivals, Zipf matrix choice
# ---------------------------------------------------------------------------

def serve_pool():
    """Eight distinct matrices (power-law and 27-point stencil styles, N from
    50K to 2M, smallest first: the Zipf choice favours the small ones); each
    is registered eight times, giving 64 resident matrices of about 20 GB in
    FP64."""
    return [M.powerlaw(50_000, seed=21), M.stencil27(100), M.powerlaw(1_500_000, seed=22),
            M.stencil27(110), M.powerlaw(2_000_000, seed=23), M.stencil27(120),
            M.powerlaw(2_000_000, seed=24), M.stencil27(126)]


def serve_leg(args, rates, seconds, precisions=(False, True), plan_serial=False):
    """The request loop over the 64-matrix pool at each offered rate (Poisson
    arrivals, Zipf(1.1) matrix choice) for each precision (False: FP64, True:
    mixed in the 8-column layout); one result dict per (precision, rate)."""
    import torch

    import spc5_b200 as S
    distinct = serve_pool()
    results = []
    for mixed in precisions:
        dt = np.float32 if mixed else np.float64
        tdt = torch.float32 if mixed else torch.float64
        mats = []
        for rep in range(8):
            for csr in distinct:
                m = S.csr_matrix(csr.rowptr, csr.colidx, csr.values.astype(dt), csr.ncols,
                                 value_type=S.F32_V8 if mixed else None)
                # default kernel choice: the length-sorted plan for the
                # power-law matrices (its single copy of the arrays serves
                # lone requests and batches alike), the row kernels for the
                # stencils
                S.CSR_to_SPC5(m, S.FORMAT_OF_R[1 if csr.name.startswith("powerlaw") else 4])
                mats.append((m, csr))
        srv = S.Server(slots=args.slots, max_k=16, mixed=mixed, plan_serial=plan_serial)
        ids = [srv.add_matrix(m) for m, _ in mats]
        resident = srv.stats()["resident_bytes"]
        xs = [torch.from_numpy(M.x_vector(csr.ncols, 500 + i, dt)).cuda() for i, csr in enumerate(distinct)]
        depth = 32  # enough outstanding outputs per matrix that arrivals never wait
        ybufs = [[torch.empty(csr.nrows, dtype=torch.float64, device="cuda") for _ in range(depth)]
                 for _, csr in mats]
        owner = [[None] * depth for _ in mats]
        # warm-up, untimed: every kernel the rates can reach is loaded once
        # (SpMV, and SpMM passes of every width: k = 15 and 16 cover them),
        # then one request per resident matrix through the request loop
        for (m, csr), x in zip(mats[:len(distinct)], xs):
            for k in (15, 16):
                X = x[:, None].expand(csr.ncols, k).contiguous()
                Y = torch.zeros(csr.nrows, k, dtype=torch.float64 if mixed else tdt, device="cuda")
                (S.SPC5_Spmm_mixed if mixed else S.SPC5_Spmm)(m, X, Y)
            del X, Y
        torch.cuda.synchronize()
        for i in range(len(mats)):
            srv.wait(srv.submit(ids[i], xs[i % len(distinct)], ybufs[i][0]))
        zipf_w = 1.0 / np.arange(1, len(mats) + 1) ** 1.1
        zipf_w /= zipf_w.sum()
        for rate in rates:
            rng = np.random.default_rng(int(rate))
            nreq = int(rate * seconds)
            arrivals = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
            choice = rng.choice(len(mats), size=nreq, p=zipf_w)
            srv.stats(reset=True)
            slot_ptr = [0] * len(mats)
            t0 = time.perf_counter()
            for t_arr, i in zip(arrivals, choice):
                while time.perf_counter() - t0 < t_arr:
                    pass
                j = slot_ptr[i]
                slot_ptr[i] = (j + 1) % depth
                if owner[i][j] is not None:
                    srv.wait(owner[i][j])
                owner[i][j] = srv.submit(ids[i], xs[i % len(distinct)], ybufs[i][j])
            srv.drain()
            for row in owner:
                for j in range(depth):
                    row[j] = None
            st = srv.stats(reset=True)
            results.append({"precision": "mixed" if mixed else "f64", "offered_req_per_s": rate,
                            "req_per_s": round(st["req_per_s"], 1), "p50_us": round(st["p50_us"], 1),
                            "p99_us": round(st["p99_us"], 1), "mean_k": round(st["mean_k"], 2),
                            "launches": st["launches"], "completed": st["completed"],
                            "resident_gb": round(resident / 1e9, 2)})
        srv.close()
        del mats, ybufs, xs
        torch.cuda.empty_cache()
    return results


def run_serve(args):
    import torch
    torch.cuda.set_device(0)
    rates = [float(t) for t in args.rates.split(",")]
    results = serve_leg(args, rates, args.serve_seconds, plan_serial=args.plan_serial)
    best = max(r["req_per_s"] for r in results if r["precision"] == "f64")
    line = {"metric": "served SpMV req/s and p50/p99 latency", "value": best, "unit": "req/s",
            "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "serve", "resident_matrices": 64,
                       "desc": "8 distinct power-law / 27-point stencil matrices (N 50K..2M), each "
                               "registered 8 times; Poisson arrivals, Zipf(1.1) matrix choice, "
                               f"coalescing up to k=16, {args.slots} slots",
                       "seconds_per_rate": args.serve_seconds},
            "serving": results}
    print(json.dumps(line))
    return 0


# DRAM bytes per algorithmic byte of one SpMV with the default kernels, per
# format, measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum
# over all launches of the call) on the same generators at smaller sizes
# (power-law N = 1M, stencil 100^3); traffic grows with the units processed,
# so roofline.traffic of the full workloads is these ratios times their bytes.
L2_BYTES = 126e6  # B200 L2

TRAFFIC_RATIO = {"powerlaw": {1: 1.199, 2: 1.203, 4: 1.168, 8: 1.593},
                 "stencil27": {1: 0.999, 2: 0.984, 4: 0.978, 8: 0.994}}

# spc5cuda_mat_kernel codes: SPC5CUDA_KERNEL_GROUPS = 1, SPC5CUDA_KERNEL_ROWS = 2
KERNEL_NAME = {1: "k_spmv (group per block-row stream)", 2: "k_rows (thread per sub-row)",
               3: "sorted plan (k_rows by block-row size; largest block-rows as multiply-add chains, k_chain_spmv)", 0: "unconverted"}


def select_kernel(m, which):
    """Apply --kernel to a converted handle."""
    import spc5_b200 as S
    if which == "groups":
        m.set_kernel(S.KERNEL_GROUPS)
    elif which == "sorted":
        m.set_kernel(S.KERNEL_SORTED)
    elif which == "rows":
        try:
            m.set_kernel(S.KERNEL_ROWS)
        except S.SPC5Error:
            m.set_kernel(S.KERNEL_AUTO)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["powerlaw", "stencil27", "poisson", "batched", "serve"],
                    default="powerlaw")
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--rates", default="5000,20000,50000", help="serving arrival rates (req/s)")
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--plan-serial", action="store_true",
                    help="serve: sorted-plan matrices run their parts in order on the slot's stream")
    ap.add_argument("--size", type=int, default=None,
                    help="smaller workload for profiling (rows for powerlaw, grid edge for stencil27)")
    ap.add_argument("--formats", default="1,2,4,8", help="comma list of r to run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--mode", choices=["replicas", "sharded"], default="replicas",
                    help="N > 1: every rank runs its own copy (replicas), or one matrix is cut into "
                         "block-row shards iterated with an NCCL all-gather of x (sharded)")
    ap.add_argument("--no-extra", action="store_true",
                    help="default run: skip the stencil, Poisson and serving legs")
    ap.add_argument("--kernel", choices=["auto", "groups", "rows", "sorted"], default="auto",
                    help="SpMV kernel (rows falls back to auto where a block-row does not fit)")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu dram bytes per launch of the dominant kernel, if captured")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global FORMATS
    FORMATS = tuple(int(t) for t in args.formats.split(","))
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.mode == "sharded":
        return run_sharded(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
