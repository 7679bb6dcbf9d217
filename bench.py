#!/usr/bin/env python
"""Benchmark of the gooseberry sparse hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

Default workload (N=1): plain FP64 conjugate gradient on the 2D 5-point
Laplacian of a 1024x1024 grid (n = 1,048,576, nnz = 5,238,784), b uniform in
[-1, 1] (seed 2), x0 = 0, stop at ||r|| <= 1e-8 ||b|| or 5000 iterations --
the reference's cgd contract (src/cgd.c:40-129).  One step = one full solve
with the matrix and b already in HBM; L2 is flushed (256 MB write) between
steps, outside the timed events.  `value` = solves/s over all ranks.

Other workloads (--workload): spmv_uniform (100k x 100k, 10 nnz/row, FP64),
spmv_powerlaw (8M rows, 128M nnz, power-law rows, FP64 and FP32).

--impl reference times the reference's own OpenMP CPU code (oracle/_ref,
else the oracle restatement) on this host's cores for the same workload and
metric, on a bounded sample of iterations per step.

Multi-GPU: the path runs on one GPU; with --gpus N (under torchrun) every rank
runs an independent replica (no data-path collective), timing is the max over
ranks and `value` sums all ranks' solves ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
PROFILES = os.path.join(ROOT, "profiles")
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, copy burst)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def cg_a_kernel_name(entry_bytes, row_bytes):
    """The FP64 CG's A kernel for the solver's matrix layout (stored bytes per
    entry and per row)."""
    if entry_bytes == 0:
        return ("cg_a_ell8_kernel (row patterns, value codes in rows of 8; SpMV + "
                "p update + p.Ap)" if row_bytes == 9 else
                "cg_a_ellv_kernel (row patterns, values in rows of 6 or 8; SpMV + "
                "p update + p.Ap)")
    if entry_bytes < 12:
        return ("cg_a_codec_kernel (row schedule over the compressed entries; SpMV + "
                "p update + p.Ap)")
    return "cg_a_kernel (SpMV + p update + p.Ap)"


def ncu_traffic(kernel_key: str):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary
    (profiles/*.txt lines `traffic_bytes_per_launch <key> <bytes> <scale>`)."""
    if not os.path.isdir(PROFILES):
        return None
    for fn in sorted(os.listdir(PROFILES)):
        if not fn.endswith(".txt"):
            continue
        with open(os.path.join(PROFILES, fn)) as f:
            for ln in f:
                parts = ln.split()
                if len(parts) >= 3 and parts[0] == "traffic_bytes_per_launch" \
                        and parts[1] == kernel_key:
                    return float(parts[2])
    return None


# ---- distributed plumbing -------------------------------------------------------

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def aggregate(self, units_local: float, t_local: float):
        """Replicas: every rank times its own units of work; the job's rate is
        all ranks' units over the slowest rank's time.  Returns (rate, t_max)."""
        t_max = self.max(t_local)
        return self.sum(units_local) / t_max, t_max

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---- clocks -----------------------------------------------------------------------

class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.err = None

    def start(self):
        try:
            import torch
            p = torch.cuda.get_device_properties(self.dev)
            sel = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:
            sel = str(self.dev)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", sel, f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception as e:  # no nvidia-smi
            self.err = str(e)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        rows = [[c.strip() for c in ln.split(",")] for ln in self.lines if ln.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "note": self.err or "no samples"}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---- workloads --------------------------------------------------------------------

def cg_laplace_setup():
    from gooseberry_b200 import workloads as W
    L = W.laplacian_2d(1024)
    b = W.rhs(L.nrows, 2)
    return L, b


REF_CG_ITERS_FALLBACK = None


def reference_cg_iterations():
    """The reference's iteration count on the full system (committed golden,
    generated by tests/golden/make_golden.py from the reference itself)."""
    p = os.path.join(ROOT, "tests", "golden", "full_sizes.json")
    try:
        with open(p) as f:
            return int(json.load(f)["cg_laplace_1024"]["iterations"])
    except Exception:
        return None


def cpu_cg_sample(L, b, rtol, iters_full, budget_s=10.0, threads=None):
    """Time the reference cgd (oracle/_ref, else the restatement) for a bounded
    number of iterations on this host; returns (solves/s, info)."""
    import oracle
    threads = threads or host_cores()
    err = rtol * float(np.linalg.norm(b))
    kind = "reference" if oracle.ref_available("f64") else "port"
    if kind == "reference":
        oracle.ref_set_threads(threads)

        def run(k):
            return oracle.ref_cgd(L.rowptr, L.rowind, L.rowval, b, err, k)
    else:
        def run(k):
            return oracle.cgd(L.rowptr, L.rowind, L.rowval, b, err, k, threads=threads)
    t0 = time.perf_counter()
    run(10)
    t_iter = (time.perf_counter() - t0) / 10
    k = int(max(20, min(iters_full, budget_s / max(t_iter, 1e-9))))
    t0 = time.perf_counter()
    _, done, _ = run(k)
    dt = time.perf_counter() - t0
    t_iter = dt / max(done, 1)
    solves = 1.0 / (t_iter * iters_full)
    return solves, {"kind": kind, "cores": threads, "iterations_timed": done,
                    "seconds": dt, "s_per_iteration": t_iter}


def run_cg_laplace(args, dist: Dist):
    import torch

    import gooseberry_b200 as gb

    dev = dist.local if torch.cuda.device_count() > dist.local else 0
    torch.cuda.set_device(dev)
    L, b = cg_laplace_setup()
    n, nnz = L.nrows, L.nnz
    rtol, niter = 1e-8, 5000
    # the default schedule for short, even rows is the row schedule, which is
    # the fastest CG SpMV measured on this matrix; the autotuner is not used
    # here because it times a plain SpMV, not the fused CG kernel
    A = gb.CsrMatrix.from_host(L)
    S = gb.CgSolver(A)
    bd = torch.from_numpy(b).cuda()
    xd = torch.empty_like(bd)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # live per-kernel timing (first iterations of a real solve)
    ms_a, ms_b = S.profile(bd, iterations=40)
    # algorithmic bytes of the A kernel in the CSR layout (rowptr, column +
    # value per nonzero, r & p gathered once, p & Ap written); the kernel
    # itself streams a lossless compressed copy of the entries when the matrix
    # allows (16-bit column distances, 8-bit codes into the table of distinct
    # values: entry_bytes = 3 instead of 12; on pattern matrices with value
    # codes nothing per entry and 9 bytes per row), reported beside it
    entry_bytes = S.entry_bytes()
    ell8 = entry_bytes == 0 and S.row_bytes() == 9  # pattern byte + 8 value codes
    bytes_a = 4 * (n + 1) + 12 * nnz + 32 * n
    bytes_a_stored = S.row_bytes() * (n + 1) + entry_bytes * nnz + 32 * n
    bytes_b = 48 * n                             # x, p, r, Ap read; x, r written
    bytes_textbook = 4 * (n + 1) + 12 * nnz + 14 * 8 * n

    for _ in range(args.warmup):
        S.solve(bd, xd, tol=rtol, relative=True, niter=niter)
    torch.cuda.synchronize()

    clocks = Clocks(dev)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    evs = []
    results = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _, r = S.solve(bd, xd, tol=rtol, relative=True, niter=niter)
        e1.record()
        evs.append((e0, e1))
        results.append(r)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    t_local = sum(a.elapsed_time(b_) for a, b_ in evs) / 1e3
    rate, t_max = dist.aggregate(float(args.steps), t_local)
    iters = results[-1].iterations
    assert all(r.status == "converged" for r in results), [r.status for r in results]

    # end to end through the drop-in C ABI, host (pinned) buffers, copies timed
    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()
    h_rp, h_ri, h_rv, h_b = pinned(L.rowptr.view(np.int32)).view(np.uint32), \
        pinned(L.rowind.view(np.int32)).view(np.uint32), pinned(L.rowval), pinned(b)
    h_x = pinned(np.zeros(n, dtype=np.float64))
    err_abs = rtol * float(np.linalg.norm(b))
    # warm-up calls as for the device timing: the second call of a process
    # still ran 3 ms slower than the later ones (68.6 against 65.1-65.5 ms)
    e2e_warm = max(1, min(args.warmup, 3))
    for _ in range(e2e_warm):
        gb.cgd(h_rp, h_ri, h_rv, h_b, err_abs, niter, out=h_x)
    e2e_steps = max(1, min(args.steps, 5))
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        xh, it_e2e, _ = gb.cgd(h_rp, h_ri, h_rv, h_b, err_abs, niter, out=h_x)
    t_e2e = dist.max(time.perf_counter() - t0)
    h2d = 4 * (n + 1) + 4 * nnz + 8 * nnz + 8 * n
    d2h = 8 * n

    peak, peak_src = hbm_peak()
    ach_a = bytes_a / (ms_a * 1e-3) / 1e9
    ach_a_stored = bytes_a_stored / (ms_a * 1e-3) / 1e9
    out = {
        "metric": "CG solves/s (FP64, 2D 5-point Laplacian 1024x1024, rel-res 1e-8)",
        "value": rate,
        "unit": "solves/s",
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_max / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded b ~ U[-1,1] (seed 2), exact 5-point Laplacian",
        "config": {
            "workload": "cg_laplace2d_1024 (plain FP64 CG, x0=0, rel-res 1e-8, max 5000 it)",
            "n": n, "nnz": nnz, "rtol": rtol, "niter": niter, "iterations": iters,
            "reference_iterations": reference_cg_iterations(),
            "schedule": gb.SCHED_NAMES[A.info().schedule],
            "tile_items": A.info().tile_items,
            "matrix_bytes_per_entry": entry_bytes,
            "matrix_bytes_per_row": S.row_bytes(),
            "l2": "flushed between steps (256 MB write, outside the timed events)",
            "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
        },
        "roofline": {
            "bound": "hbm",
            "kernel": cg_a_kernel_name(entry_bytes, S.row_bytes()),
            "achieved": ach_a, "peak": peak, "unit": "GB/s", "frac": ach_a / peak,
            "traffic": ncu_traffic("cg_a_ell8_laplace1024" if ell8
                                   else "cg_a_ellv_laplace1024" if entry_bytes == 0
                                   else "cg_a_codec_laplace1024" if entry_bytes < 12
                                   else "cg_a_row_laplace1024"),
            "bytes_per_launch": bytes_a, "launch_ms": ms_a, "peak_source": peak_src,
            "bytes_per_launch_stored": bytes_a_stored,
            "achieved_stored": ach_a_stored, "frac_stored": ach_a_stored / peak,
            # one iteration's working set (stored matrix + vectors) fits in
            # the 126 MB L2, which the solve keeps it in (evict-last hints):
            # the kernel's bytes mostly come from L2, not HBM
            "l2_resident": bool(bytes_a_stored + 16 * n <= 126e6),
            "frac_textbook_per_step": (bytes_textbook * iters * args.steps / t_local / 1e9)
                                      / peak,
        },
        "kernels": {
            "cg_a_ms": ms_a, "cg_b_ms": ms_b,
            "cg_b_gbs": bytes_b / (ms_b * 1e-3) / 1e9,
            "iteration_ms": (t_local / args.steps) / iters * 1e3,
            "iteration_fused_gbs": (bytes_a + bytes_b) * iters * args.steps / t_local / 1e9,
            "iteration_textbook_gbs": bytes_textbook * iters * args.steps / t_local / 1e9,
            "bytes_per_iteration_fused": bytes_a + bytes_b,
            "bytes_per_iteration_stored": bytes_a_stored + bytes_b,
            "bytes_per_iteration_textbook": bytes_textbook,
        },
        "e2e": {"value": e2e_steps * dist.world / t_e2e, "unit": "solves/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "gooseberry_cgd_f64 (host pinned buffers)", "iterations": it_e2e,
                "calls": e2e_steps, "warmup_calls": e2e_warm},
        "gpu_launches": int(sum(r.kernel_launches for r in results)),
        "clocks": clk,
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        ref_it = reference_cg_iterations() or iters
        v, info = cpu_cg_sample(L, b, rtol, ref_it)
        out["cpu_baseline"] = {
            "value": v, "unit": "solves/s", "cores": info["cores"], "kind": info["kind"],
            "sample": (f"{info['iterations_timed']} of the {ref_it} iterations of one solve "
                       f"({info['seconds']:.1f} s, {info['s_per_iteration'] * 1e3:.2f} ms/it), "
                       "scaled to a full solve"),
        }
    return out


def _spmv_bytes(n, nnz, s_v, s_x):
    # 4(n+1) rowptr + nnz (index + value) + x once + y once
    return 4 * (n + 1) + nnz * (4 + s_v) + n * s_x + n * s_x


def _cond_err(y, y_ref, A, x):
    import scipy.sparse as sp
    S = sp.csr_matrix((np.abs(A.rowval), A.rowind.astype(np.int64),
                       A.rowptr.astype(np.int64)), shape=(A.nrows, A.ncols))
    scale = S @ np.abs(x.astype(np.float64))
    return float(np.max(np.abs(y.astype(np.float64) - y_ref) / np.maximum(scale, 1e-300)))


def measure_spmv(A, x, reps=20, f32=False, flush=None, schedule=None):
    """Device time of one SpMV (CUDA events, L2 flushed before each rep).
    Returns (ms, y, info)."""
    import torch

    import gooseberry_b200 as gb
    M = gb.CsrMatrix.from_host(A, f64=not f32, f32=f32)
    if schedule is None:
        M.autotune(f32=f32)
    else:
        M.set_schedule(schedule, f32=f32)
    xd = torch.from_numpy(x.astype(np.float32 if f32 else np.float64)).cuda()
    y = M.spmv(xd)
    for _ in range(3):
        M.spmv(xd, y)
    times = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        M.spmv(xd, y)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    info = M.info()
    sched = gb.SCHED_NAMES[info.schedule_f32 if f32 else info.schedule]
    return float(np.median(times)), y.cpu().numpy(), {"schedule": sched,
                                                      "tile_items": info.tile_items,
                                                      "nlong": info.nlong}


def measure_spdot(A, x, reps=20, f32=False, flush=None):
    """Device time of gb_spdot over the matrix's own (rowind, rowval) and x: it
    streams the same bytes and gathers the same x entries as the SpMV, without
    the row reductions and the y writes -- a floor for the SpMV on this GPU.
    Timed through the C-ABI with a preallocated result (no host sync inside)."""
    import torch

    import gooseberry_b200 as gb
    dt = np.float32 if f32 else np.float64
    ind = torch.from_numpy(A.rowind.astype(np.int32)).cuda()
    val = torch.from_numpy(A.rowval.astype(dt)).cuda()
    xd = torch.from_numpy(x.astype(dt)).cuda()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    fn = gb.lib().gb_spdot_f32 if f32 else gb.lib().gb_spdot_f64
    stream = torch.cuda.current_stream().cuda_stream

    def run():
        rc = fn(A.nnz, ind.data_ptr(), val.data_ptr(), xd.data_ptr(), A.ncols,
                out.data_ptr(), stream)
        if rc != 1:
            raise RuntimeError(gb.last_error())
    for _ in range(3):
        run()
    times = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    del ind, val, xd
    return float(np.median(times))


def spmv_extra(name, A, x, peak, flush, rows_check=200_000):
    """SpMV GB/s for one matrix, FP64 and FP32.  CPU baseline: the reference's
    blas_spmult (FP64) on the first `rows_check` rows, a bounded sample on all
    host threads; its result there is also the parity check of both widths."""
    out = {"n": A.nrows, "nnz": A.nnz}
    k = min(rows_check, A.nrows)
    nnz_k = int(A.rowptr[k])
    sub = type(A)(k, A.ncols, A.rowptr[: k + 1], A.rowind[:nnz_k], A.rowval[:nnz_k])
    v, cinfo, y_ref = cpu_spmv_sample(sub, x, _spmv_bytes(k, nnz_k, 8, 8), budget_s=1.0)
    out["cpu_baseline"] = {"value": v, "unit": "GB/s", "cores": cinfo["cores"],
                           "kind": cinfo["kind"],
                           "sample": f"first {k} rows: {cinfo['sample']}"}
    for f32 in (False, True):
        ms, y, info = measure_spmv(A, x, f32=f32, flush=flush)
        b = _spmv_bytes(A.nrows, A.nnz, 4 if f32 else 8, 4 if f32 else 8)
        gbs = b / (ms * 1e-3) / 1e9
        floor = measure_spdot(A, x, f32=f32, flush=flush)
        out["f32" if f32 else "f64"] = {
            "ms": ms, "GB/s": gbs, "frac_of_peak": gbs / peak, "bytes": b, **info,
            "working_set_fits_l2": bool(b <= 126e6), "l2": "flushed before every rep",
            "max_cond_err_vs_fp64_reference_first_rows": _cond_err(y[:k], y_ref, sub, x),
            "stream_gather_floor_ms": floor, "frac_of_floor": floor / ms,
        }
    return out


def run_spmv(args, dist: Dist, which: str):
    """--workload spmv_uniform | spmv_powerlaw: SpMV GB/s (FP64 headline)."""
    import torch

    import gooseberry_b200 as gb
    from gooseberry_b200 import workloads as W
    dev = dist.local if torch.cuda.device_count() > dist.local else 0
    torch.cuda.set_device(dev)
    if which == "spmv_uniform":
        A = W.uniform_rows(100_000, 10, seed=1)
        x = W.dense_x(A.ncols, 1)
        label = "uniform 100k x 100k, 10 nnz/row"
    else:
        A = W.powerlaw_rows(8_000_000, 128_000_000, seed=3, cap=200_000)
        x = W.dense_x(A.ncols, 3)
        label = "power-law rows 8M x 8M, 128M nnz, exponent 2.1, cap 200k"
    n, nnz = A.nrows, A.nnz
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    peak, peak_src = hbm_peak()
    M = gb.CsrMatrix.from_host(A)
    M.autotune()
    xd = torch.from_numpy(x).cuda()
    y = M.spmv(xd)
    for _ in range(args.warmup):
        M.spmv(xd, y)
    clocks = Clocks(dev)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        M.spmv(xd, y)
        e1.record()
        times.append((e0, e1))
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    t_local = sum(a.elapsed_time(b) for a, b in times) / 1e3
    b = _spmv_bytes(n, nnz, 8, 8)
    rate, t_max = dist.aggregate(args.steps * b / 1e9, t_local)
    ms = t_local / args.steps * 1e3
    y_host = y.cpu().numpy()
    floor_ms = measure_spdot(A, x, flush=flush)
    # end to end: gooseberry_spmult_f64 with pinned host buffers
    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        t.numpy()[...] = a
        return t.numpy()
    h_rp = pinned(A.rowptr.view(np.int32)).view(np.uint32)
    h_ri = pinned(A.rowind.view(np.int32)).view(np.uint32)
    h_rv, h_x = pinned(A.rowval), pinned(x)
    h_y = pinned(np.zeros(n))
    gb.spmult(h_rp, h_ri, h_rv, h_x, out=h_y)
    e2e_steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        gb.spmult(h_rp, h_ri, h_rv, h_x, out=h_y)
    t_e2e = dist.max(time.perf_counter() - t0)
    info = M.info()
    out = {
        "metric": f"SpMV GB/s (FP64, {label})",
        "value": rate,
        "unit": "GB/s", "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic, seeded (gooseberry_b200.workloads)",
        "config": {"workload": which, "n": n, "nnz": nnz, "bytes_per_spmv": b,
                   "schedule": gb.SCHED_NAMES[info.schedule], "tile_items": info.tile_items,
                   "long_rows": info.nlong, "max_row": info.max_row,
                   "l2": "flushed before every SpMV (256 MB write, outside the events)"},
        "roofline": {"bound": "hbm", "kernel": "spmv_tiles_kernel",
                     "achieved": b / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": b / (ms * 1e-3) / 1e9 / peak, "traffic": ncu_traffic(which),
                     "peak_source": peak_src,
                     "stream_gather_floor_ms": floor_ms,
                     "frac_of_stream_gather_floor": floor_ms / ms},
        "e2e": {"value": e2e_steps * b / t_e2e / 1e9, "unit": "GB/s",
                "h2d_bytes_per_step": 4 * (n + 1) + 12 * nnz + 8 * n,
                "d2h_bytes_per_step": 8 * n, "api": "gooseberry_spmult_f64 (pinned host)"},
        "gpu_launches": args.steps, "clocks": clk,
    }
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        v, cinfo, y_ref = cpu_spmv_sample(A, x, b)
        out["cpu_baseline"] = {"value": v, "unit": "GB/s", "cores": cinfo["cores"],
                               "kind": cinfo["kind"], "sample": cinfo["sample"]}
        # the baseline's result is the parity check (first 200k rows)
        k = min(200_000, n)
        nnz_k = int(A.rowptr[k])
        sub = type(A)(k, A.ncols, A.rowptr[: k + 1], A.rowind[:nnz_k], A.rowval[:nnz_k])
        out["config"]["parity_max_cond_err_first_200k_rows"] = _cond_err(
            y_host[:k], y_ref[:k], sub, x)
    return out


def cpu_spmv_sample(A, x, nbytes, budget_s=10.0):
    """The reference's blas_spmult (oracle/_ref, else the restatement) on all
    host threads; GB/s over repeated full SpMVs within the time budget.
    Returns (GB/s, info, y) with y the baseline's own result."""
    import oracle
    threads = host_cores()
    kind = "reference" if oracle.ref_available("f64") else "port"
    if kind == "reference":
        oracle.ref_set_threads(threads)
        run = lambda: oracle.ref_spmm(A.rowptr, A.rowind, A.rowval, x, ncols=A.ncols)  # noqa: E731
    else:
        run = lambda: oracle.spmv(A.rowptr, A.rowind, A.rowval, x, threads=threads)  # noqa: E731
    y = run()
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < budget_s or reps == 0:
        run()
        reps += 1
        if reps >= 1000:
            break
    dt = time.perf_counter() - t0
    return reps * nbytes / dt / 1e9, {"kind": kind, "cores": threads,
                                      "sample": f"{reps} full SpMVs in {dt:.1f} s"}, y


def _reference_cg_solution(side):
    """The reference cgd's solution on the 160^3 operator (every step-th entry)
    and its golden record, from tests/golden (made by running the reference's
    own build); None for other sizes."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden")
    try:
        with open(os.path.join(path, "full_sizes.json")) as f:
            g = json.load(f)["cg_diffusion_160"]
        xs = np.load(os.path.join(path, "cg_diffusion_160_xsample.npz"))
    except (OSError, KeyError):
        return None
    if g["side"] != side:
        return None
    return g, int(xs["step"]), xs["x"]


def mixed_extra(side=160, rtol=1e-10, reps=2, peak=None):
    """Mixed-precision CG (FP32 inner, FP64 refinement) against plain FP64 CG
    on the 3D 7-point variable-coefficient operator (160^3, coefficients
    log-uniform in [1e-2, 1e2]); errors are true FP64 residuals on the host
    and distances to the reference cgd's solution (tests/golden).  Per-kernel
    device times come from the solver's profiler (launch by launch, CUDA
    events); the FP64 solver's SpMV kernel gets a roofline block: its bytes in
    CSR terms (4(n+1) + 12 nnz + 32 n: rowptr, entries, r and p gathered once,
    p and Ap written) and in the bytes it stores per entry."""
    import torch

    import gooseberry_b200 as gb
    from gooseberry_b200 import workloads as W
    A = W.diffusion_3d(side, seed=4)
    b = W.rhs(A.nrows, 4)
    n, nnz = A.nrows, A.nnz
    M = gb.CsrMatrix.from_host(A, f64=True, f32=True)
    bd = torch.from_numpy(b).cuda()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    S_ = A.to_scipy()
    ref = _reference_cg_solution(side)
    out = {"n": n, "nnz": nnz, "rtol": rtol,
           "l2": "flushed before each timed solve (256 MB write)"}
    if ref is not None:
        out["reference"] = {"iterations_by_omp_threads": ref[0]["reference_iterations_by_threads"],
                            "solution": f"every {ref[1]}-th entry of the reference cgd's x"}
    for name, mode in (("f64", gb.CG_F64), ("mixed", gb.CG_MIXED)):
        S = gb.CgSolver(M, mode=mode)
        x, r = S.solve(bd, tol=rtol, niter=50000)
        ts = []
        for _ in range(reps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            x, r = S.solve(bd, tol=rtol, niter=50000)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        xh = x.cpu().numpy()
        rel = float(np.linalg.norm(b - S_ @ xh) / np.linalg.norm(b))
        prof = S.profile(bd, iterations=20)
        names = (["spmv_direction_pap", "x_r_update_rr"] if mode == gb.CG_F64 else
                 ["spmv32_direction_pap", "y_r_update_rr", "fp64_residual_of_a_refinement"])
        d = {"ms": min(ts), "solves_per_s": 1e3 / min(ts), "iterations": r.iterations,
             "refinements": r.refinements, "status": r.status, "true_rel_residual": rel,
             "us_per_iteration": 1e3 * min(ts) / max(r.iterations, 1),
             "kernels_us": {k: 1e3 * v for k, v in zip(names, prof)},
             "kernel_launches": r.kernel_launches,
             "entry_bytes": S.entry_bytes(), "row_bytes": S.row_bytes(),
             "schedule": gb.SCHED_NAMES[
                 M.info().schedule_f32 if mode == gb.CG_MIXED else M.info().schedule]}
        if ref is not None:
            d["rel_err_vs_reference_solution"] = float(
                np.linalg.norm(xh[::ref[1]] - ref[2]) / np.linalg.norm(ref[2]))
        if mode == gb.CG_F64:
            x64 = xh
            if peak:
                eb, rb = S.entry_bytes(), S.row_bytes()
                a_ms = prof[0]
                bytes_csr = 4 * (n + 1) + 12 * nnz + 32 * n
                bytes_stored = rb * (n + 1) + eb * nnz + 32 * n
                d["roofline"] = {
                    "bound": "hbm", "kernel": cg_a_kernel_name(eb, rb),
                    "launch_ms": a_ms, "bytes_per_launch": bytes_csr,
                    "achieved": bytes_csr / (a_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                    "frac": bytes_csr / (a_ms * 1e-3) / 1e9 / peak,
                    "bytes_per_launch_stored": bytes_stored,
                    "frac_stored": bytes_stored / (a_ms * 1e-3) / 1e9 / peak,
                    "l2_resident": False}
        else:
            d["rel_diff_to_fp64_solution"] = float(np.linalg.norm(xh - x64) / np.linalg.norm(x64))
            if peak:
                # A32: FP32 values, r and p gathered (4 B each per row), p_new and
                # Ap written; stored bytes per the solver's layout (rows of 8
                # padded values and a pattern byte on stencils)
                eb, rb = S.entry_bytes(), S.row_bytes()
                a_ms = prof[0]
                bytes_csr = 4 * (n + 1) + 8 * nnz + 16 * n
                bytes_stored = rb * (n + 1) + eb * nnz + 16 * n
                d["roofline"] = {
                    "bound": "hbm", "kernel": "A32 (FP32 SpMV + p update + p.Ap in FP64)",
                    "launch_ms": a_ms, "bytes_per_launch": bytes_csr,
                    "achieved": bytes_csr / (a_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                    "frac": bytes_csr / (a_ms * 1e-3) / 1e9 / peak,
                    "bytes_per_launch_stored": bytes_stored,
                    "frac_stored": bytes_stored / (a_ms * 1e-3) / 1e9 / peak,
                    "l2_resident": False}
        out[name] = d
        S.close()
    out["speedup_mixed_over_f64"] = out["f64"]["ms"] / out["mixed"]["ms"]
    return out


def _serve_live(srv, reqs, arr, rtol, limit_s=3600.0):
    """Drive a server in real time: request i is submitted at arr[i] seconds
    after the start; returns the results and their latencies (arrival to
    result, seconds, on the server's clock)."""
    n = len(reqs)
    c0 = srv.clock()
    i, got = 0, []
    t_start = time.perf_counter()
    while len(got) < n and time.perf_counter() - t_start < limit_s:
        now = time.perf_counter() - t_start
        while i < n and arr[i] <= now:
            srv.submit(i, reqs[i][1], reqs[i][2], tol=rtol)
            i += 1
        active, queued = srv.step()
        got += srv.poll()
        if active == 0 and queued == 0 and i < n:
            time.sleep(max(0.0, min(0.01, arr[i] - (time.perf_counter() - t_start))))
    return got, [r.t_done - c0 - arr[r.id] for r in got]


def _serve_saturated(srv, reqs, rtol, depth, limit_s=3600.0):
    """Every request is there at t = 0; the loop keeps `depth` of them queued
    ahead of the device and submits the rest between steps, so the host's copy
    of a request overlaps the device work of the ones before it."""
    n = len(reqs)
    i, got, queued = 0, [], 0
    t_start = time.perf_counter()
    while len(got) < n and time.perf_counter() - t_start < limit_s:
        while i < n and queued < depth:
            k, A, b = reqs[i]
            srv.submit(k, A, b, tol=rtol)
            i += 1
            queued += 1
        _, queued = srv.step()
        got += srv.poll()
    return got


def serving_extra(nreq=300, seed=5, rtol=1e-10, pool=16 << 30, slots=256, ips=16,
                  load=0.8, live=True, dropin=True, arm_names=None):
    """Serving stream of 2D 5-point variable-coefficient SPD systems (side
    log-uniform in [32, 512], coefficients log-uniform in [0.1, 10], b in
    [-1, 1], per-request seeds), each to rel-res `rtol`.

    Server arms on the same stream (16 GB pool, `ips` iterations per step):
      mixed_batched      continuous batching, FP32 inner iterations with FP64
                         refinement, up to `slots` solves resident;
      fp64_batched       the same server in plain FP64 CG;
      fp64_one_at_a_time the same server in FP64 with one slot: plain FP64 CG
                         served one solve at a time (the benchmark's baseline).
    Each arm: the saturated rate (every request present at t = 0 and kept
    queued two slot-counts deep ahead of the device, after an untimed pass that
    grows the server to its working size), then a live run
    under Poisson arrivals at `load` x the one-at-a-time arm's saturated rate,
    the same arrival times for every arm, with p50/p99 latency from arrival
    to result.  For context (streams of up to 1000 requests), the drop-in
    gooseberry_cgd_f64 (upload, solve, download per request) one at a time
    at saturation.  Each server's stats (device time of its graph replays,
    host time per step and in submit, tile autotuner runs) come with it."""
    import gooseberry_b200 as gb
    from gooseberry_b200 import workloads as W
    sides = W.serving_sides(nreq, seed)
    reqs = []
    for k, side in enumerate(sides):
        rs = seed * 1_000_003 + k
        A = W.diffusion_2d(int(side), seed=rs)
        reqs.append((k, A, W.rhs(A.nrows, rs)))

    def pct(v, q):
        return float(np.percentile(np.asarray(v), q)) if len(v) else None

    arms = {"mixed_batched": (gb.CG_MIXED, slots), "fp64_batched": (gb.CG_F64, slots),
            "fp64_one_at_a_time": (gb.CG_F64, 1)}
    if arm_names:
        arms = {k: v for k, v in arms.items() if k in arm_names}
    servers, out = {}, {}
    for name, (mode, ns) in arms.items():
        srv = gb.Server(pool_bytes=pool, max_slots=ns, mode=mode, iters_per_step=ips)
        # the warm pass: the whole stream for a batched server up to 1000
        # requests (it reaches full residency), else every 10th request
        warm = reqs if ns > 1 and nreq <= 1000 else reqs[::10]
        for k, A, b in warm:
            srv.submit(k, A, b, tol=rtol)
        srv.drain(timeout_s=3600)
        t0 = time.perf_counter()
        res = _serve_saturated(srv, reqs, rtol, depth=2 * ns)
        makespan = time.perf_counter() - t0
        worst = 0.0
        for r in res:
            A, b = reqs[r.id][1], reqs[r.id][2]
            worst = max(worst, float(np.linalg.norm(b - A.to_scipy() @ r.x) /
                                     np.linalg.norm(b)))
        out[name] = {"solves_per_s_saturated": len(res) / makespan,
                     "server_stats_saturated": srv.stats(),
                     "converged": sum(r.status == "converged" for r in res),
                     "worst_true_rel_residual": worst,
                     "iterations_median": float(np.median([r.iterations for r in res]))}
        servers[name] = srv
    lam = None
    if live and "fp64_one_at_a_time" in out:
        lam = load * out["fp64_one_at_a_time"]["solves_per_s_saturated"]
        arr = W.poisson_arrivals(nreq, lam, seed)
        for name, srv in servers.items():
            got, lat = _serve_live(srv, reqs, arr, rtol)
            out[name].update({"p50_s": pct(lat, 50), "p99_s": pct(lat, 99),
                              "completed_live": len(got),
                              "converged_live": sum(r.status == "converged" for r in got)})
    for srv in servers.values():
        srv.close()
    if dropin and nreq <= 1000:  # context: the drop-in, one request at a time
        for k, A, b in sorted(reqs, key=lambda q: q[1].nrows)[::10]:
            gb.cgd(A.rowptr, A.rowind, A.rowval, b, rtol * float(np.linalg.norm(b)), 0)
        t0 = time.perf_counter()
        ok = 0
        for k, A, b in reqs:
            x, it, rn = gb.cgd(A.rowptr, A.rowind, A.rowval, b,
                               rtol * float(np.linalg.norm(b)), 0)
            ok += int(rn <= rtol * float(np.linalg.norm(b)) * (1 + 1e-12))
        out["fp64_dropin_one_at_a_time"] = {"solves_per_s": nreq / (time.perf_counter() - t0),
                                            "converged": ok}

    def ratio(a, b):
        return (out[a]["solves_per_s_saturated"] / out[b]["solves_per_s_saturated"]
                if a in out and b in out else None)
    return {
        "requests": nreq, "rtol": rtol, "pool_bytes": pool, "slots": slots,
        "iters_per_step": ips,
        "rows_min_median_max": [int(min(sides) ** 2), int(np.median(sides) ** 2),
                                int(max(sides) ** 2)],
        **out,
        "arrival_rate_per_s": lam,
        "speedup_mixed_batched_over_fp64_one_at_a_time":
            ratio("mixed_batched", "fp64_one_at_a_time"),
        "speedup_mixed_batched_over_fp64_batched": ratio("mixed_batched", "fp64_batched"),
        "speedup_fp64_batched_over_fp64_one_at_a_time":
            ratio("fp64_batched", "fp64_one_at_a_time"),
    }


def spmm_extra(k=8, flush=None, peak=None, reps=20):
    """C = A B with k right-hand sides on the 2D 5-point Laplacian 1024^2 (the
    CG configuration's matrix): the fused kernel (A read once, B transposed
    row-major) against k separate SpMVs.  Algorithmic bytes: A once, B and C
    once each: 4(n+1) + 12 nnz + 16 n k."""
    import torch

    import gooseberry_b200 as gb
    from gooseberry_b200 import workloads as W
    L = W.laplacian_2d(1024)
    n, nnz = L.nrows, L.nnz
    M = gb.CsrMatrix.from_host(L)
    M.set_schedule(gb.SCHED_ROW)
    B = torch.from_numpy(np.random.default_rng(8).uniform(-1, 1, n * k)).cuda()
    C = M.spmm(B, k)
    y = torch.empty(n, dtype=torch.float64, device="cuda")

    def timed(fn):
        for _ in range(3):
            fn()
        ts = []
        for _ in range(reps):
            if flush is not None:
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))
    t_fused = timed(lambda: M.spmm(B, k, out=C))
    t_cols = timed(lambda: [M.spmv(B[j * n:(j + 1) * n], y) for j in range(k)])
    b = 4 * (n + 1) + 12 * nnz + 16 * n * k
    out = {"k": k, "n": n, "nnz": nnz, "fused_ms": t_fused, "per_column_spmv_ms": t_cols,
           "speedup": t_cols / t_fused, "GB/s": b / (t_fused * 1e-3) / 1e9,
           "bytes": b}
    if peak:
        out["frac_of_peak"] = out["GB/s"] / peak
    M.close()
    return out


def _device_spmv_ms(M, xd, flush, reps=20):
    """Median device time of one autotuned FP64 SpMV of a device matrix."""
    import torch

    import gooseberry_b200 as gb
    M.autotune()
    y = M.spmv(xd)
    for _ in range(3):
        M.spmv(xd, y)
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        M.spmv(xd, y)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return {"ms": float(np.median(ts)), "schedule": gb.SCHED_NAMES[M.info().schedule]}


def rcm_extra(powerlaw=None, flush=None):
    """Bandwidth-reducing reorder (Cuthill-McKee, src/permute.c:288-337; the
    CLI's `permute -p bandwidth` and `blas -b`).  Ours: the drop-in
    gooseberry_permute_cuthillmckee on host arrays (upload, device ordering,
    download) and the device-resident gb_csr_cuthillmckee; reference: its own
    permute.c on one host core (the unblocked call is serial), same graphs,
    equal orders required.  Then what the order buys the SpMV: the power-law
    matrix and a 2D Laplacian whose numbering was scrambled, each timed
    before and after P A P^T."""
    import torch

    import gooseberry_b200 as gb
    import oracle
    from gooseberry_b200 import workloads as W
    graphs = [("uniform_100k", W.uniform_rows(100_000, 10, seed=1)),
              ("laplace_1024", W.laplacian_2d(1024))]
    if powerlaw is not None:
        graphs.append(("powerlaw_8m", powerlaw))
    out = {}
    for name, A in graphs:
        gb.cuthillmckee(A.rowptr, A.rowind, A.nrows)  # warm
        t0 = time.perf_counter()
        perm = gb.cuthillmckee(A.rowptr, A.rowind, A.nrows)
        t_drop = time.perf_counter() - t0
        M = gb.CsrMatrix.from_host(A)
        M.cuthillmckee()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dperm = M.cuthillmckee()
        torch.cuda.synchronize()
        t_dev = time.perf_counter() - t0
        r = {"n": A.nrows, "nnz": A.nnz, "dropin_ms": t_drop * 1e3, "device_ms": t_dev * 1e3}
        if oracle.ref_available("f64"):
            t0 = time.perf_counter()
            rc, ref = oracle.ref_cuthillmckee(A.rowptr, A.rowind, A.nrows)
            t_ref = time.perf_counter() - t0
            r.update({"reference_ms": t_ref * 1e3, "reference_cores": 1,
                      "speedup_dropin_vs_reference": t_ref / t_drop,
                      "same_order_as_reference": bool(np.array_equal(perm, ref)) and bool(
                          np.array_equal(dperm.cpu().numpy().astype(np.uint32), ref))})
        if name == "powerlaw_8m":
            xd = torch.from_numpy(W.dense_x(A.nrows, 3)).cuda()
            R = M.permute(dperm, dperm)
            px = gb.permute_vector(xd, dperm)
            r["spmv_f64_before"] = _device_spmv_ms(M, xd, flush)
            r["spmv_f64_after"] = _device_spmv_ms(R, px, flush)
            R.close()
        M.close()
        out[name] = r
    # a mesh with a scrambled numbering: the order gives its locality back
    L = W.laplacian_2d(2048)
    M = gb.CsrMatrix.from_host(L)
    sp = torch.from_numpy(np.argsort(W.rand_u64(9, 30, 0, L.nrows), kind="stable")
                          .astype(np.int32)).cuda()
    S = M.permute(sp, sp)
    S.cuthillmckee()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    p = S.cuthillmckee()
    torch.cuda.synchronize()
    t_dev = time.perf_counter() - t0
    R = S.permute(p, p)
    xd = torch.from_numpy(W.dense_x(L.nrows, 4)).cuda()
    out["laplace_2048_scrambled"] = {
        "n": L.nrows, "nnz": L.nnz, "device_ms": t_dev * 1e3,
        "spmv_f64_natural": _device_spmv_ms(M, xd, flush),
        "spmv_f64_scrambled": _device_spmv_ms(S, xd, flush),
        "spmv_f64_reordered": _device_spmv_ms(R, xd, flush)}
    for X in (R, S, M):
        X.close()
    return out


def loader_extra(n=2_000_000, nnz=32_000_000, seed=9):
    """CSR text loader: a power-law matrix written in the reference's CSR
    format (%g values), then read by gooseberry_read_sparse_matrix_f64 (all
    host threads) and by gb_csr_read (parse + upload to a device matrix),
    against the reference's own single-threaded reader (src/io.c) on the same
    file."""
    import shutil
    import tempfile

    import gooseberry_b200 as gb
    import oracle
    from gooseberry_b200 import workloads as W
    A = W.powerlaw_rows(n, nnz, seed=seed, cap=200_000)
    d = tempfile.mkdtemp(prefix="gb_loader_")
    try:
        path = os.path.join(d, "a.csr")
        t0 = time.perf_counter()
        gb.write_csr(path, A.rowptr, A.rowind, A.rowval, A.ncols)
        t_write = time.perf_counter() - t0
        size = os.path.getsize(path)
        t0 = time.perf_counter()
        rp, ri, rv, nc = gb.read_csr(path)
        t_read = time.perf_counter() - t0
        # the device (context, modules) is brought up before the clock starts,
        # as it is when the loader runs after the other workloads
        gb.CsrMatrix.from_host(W.uniform_rows(1000, 10, seed=1)).close()
        t0 = time.perf_counter()
        M = gb.CsrMatrix.read(path)
        t_dev = time.perf_counter() - t0
        M.close()
        out = {"rows": n, "nnz": nnz, "file_bytes": size, "threads": os.cpu_count(),
               "write_s": t_write, "read_s": t_read, "read_to_device_s": t_dev,
               "read_GB/s": size / t_read / 1e9}
        if oracle.ref_available("f64"):
            t0 = time.perf_counter()
            rc, rn, rnc, rrp, rri, rrv = oracle.ref_read_csr(path)
            t_ref = time.perf_counter() - t0
            out["reference_read_s"] = t_ref
            out["speedup_vs_reference_read"] = t_ref / t_read
            out["same_arrays_as_reference"] = bool(
                rc == 1 and rnc == nc and np.array_equal(rrp, rp) and np.array_equal(rri, ri)
                and np.array_equal(rrv, rv))
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


def pagerank_extra(n=2_000_000, nnz=32_000_000, seed=7, tol=1e-10, cpu_iters=5):
    """PageRank (the reference's pagerank command) on a power-law directed graph
    (n nodes, nnz weighted edges, Zipf-2.1 out-degrees, weights |U[-1,1]| + 0.1),
    damping 0.85, to a change of at most `tol`.  Ours: gooseberry_pagerank_f64
    end to end (host normalisation as the reference, upload, device iterations,
    download).  CPU: the reference's loop (blas_spmult etc., all host threads) on
    a bounded sample of `cpu_iters` iterations, scaled to the same count."""
    import gooseberry_b200 as gb
    import oracle
    from gooseberry_b200 import workloads as W
    A = W.powerlaw_rows(n, nnz, seed=seed, cap=200_000)
    rv = np.abs(A.rowval) + 0.1
    gb.pagerank(A.rowptr, A.rowind, rv, 0.85, 0.0, 2)  # warm
    t0 = time.perf_counter()
    r, it, err = gb.pagerank(A.rowptr, A.rowind, rv, 0.85, tol, 0)
    t_ours = time.perf_counter() - t0
    out = {"n": n, "nnz": nnz, "tol": tol, "iterations": it, "error": err,
           "ms": t_ours * 1e3, "solves_per_s": 1.0 / t_ours,
           "rank_sum": float(r.sum())}
    if oracle.ref_available("f64"):
        threads = host_cores()
        oracle.ref_set_threads(threads)
        t0 = time.perf_counter()
        r5, _, _ = oracle.ref_pagerank(A.rowptr, A.rowind, rv, 0.85, 0.0, cpu_iters)
        t_cpu = time.perf_counter() - t0
        g5, _, _ = gb.pagerank(A.rowptr, A.rowind, rv, 0.85, 0.0, cpu_iters)
        out["cpu_reference"] = {"cores": threads, "sample_iterations": cpu_iters,
                                "sample_s": t_cpu,
                                "ms_scaled_to_iterations": t_cpu / cpu_iters * it * 1e3}
        out["max_rel_diff_vs_reference_at_sample"] = float(
            np.max(np.abs(g5 - r5)) / np.max(np.abs(r5)))
    return out


def run_extras(args):
    """Secondary workloads of the benchmark spec, reported beside the headline."""
    import torch

    from gooseberry_b200 import workloads as W
    peak, _ = hbm_peak()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    ex = {}
    t0 = time.time()
    A = W.uniform_rows(100_000, 10, seed=1)
    ex["spmv_uniform_100k"] = spmv_extra("spmv_uniform", A, W.dense_x(A.ncols, 1), peak, flush)
    A = W.powerlaw_rows(8_000_000, 128_000_000, seed=3, cap=200_000)
    ex["spmv_powerlaw_8m"] = spmv_extra("spmv_powerlaw", A, W.dense_x(A.ncols, 3), peak, flush)
    ex["rcm_reorder"] = rcm_extra(A, flush)
    del A
    # banded operators larger than L2, where x is gathered locally: the SpMV
    # kernels' streaming rate without the random-gather floor of the power-law
    # matrix (the 5-point Laplacian of a 4096^2 grid, 1.34 GB per SpMV)
    A = W.laplacian_2d(4096)
    ex["spmv_laplace_4096"] = spmv_extra("spmv_laplace_4096", A, W.dense_x(A.ncols, 4), peak,
                                         flush)
    del A
    ex["mixed_cg_3d_160"] = mixed_extra(peak=peak)
    ex["serving_stream"] = serving_extra(nreq=args.requests)
    ex["spmm_laplace1024_k8"] = spmm_extra(flush=flush, peak=peak)
    ex["pagerank_powerlaw_2m"] = pagerank_extra()
    ex["csr_loader_2m"] = loader_extra()
    ex["seconds"] = time.time() - t0
    return ex


def host_cores() -> int:
    """Physical cores of this host (logical CPUs when that cannot be read)."""
    try:
        import psutil
        return int(psutil.cpu_count(logical=False) or os.cpu_count() or 1)
    except Exception:
        return os.cpu_count() or 1


def pin_openmp() -> None:
    """OpenMP placement for the reference's CPU code: one thread per physical
    core, kept close.  Must run before the reference library is loaded (libgomp
    reads these at start-up).  Only the reference arm sets it: with
    OMP_PROC_BIND set, libgomp binds the process's main thread to the first
    core when it starts, and every host thread the library later starts from
    that thread (tile planner, text loaders) inherits that one core."""
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")


def run_reference_cg(args):
    """The reference's own cgd on all physical host cores.  A step is one
    timed block of `block` iterations of a fresh solve (x0 = 0), about 1.5 s,
    so ms_per_step x steps is the time the arm really spent; the rate is the
    block's time per iteration scaled to the reference's full iteration count
    (CG iterations cost the same from the first to the last)."""
    import oracle
    L, b = cg_laplace_setup()
    ref_it = reference_cg_iterations() or 2966
    cores = host_cores()
    err = 1e-8 * float(np.linalg.norm(b))
    kind = "reference" if oracle.ref_available("f64") else "port"
    if kind == "reference":
        oracle.ref_set_threads(cores)

        def run(k):
            return oracle.ref_cgd(L.rowptr, L.rowind, L.rowval, b, err, k)
    else:
        def run(k):
            return oracle.cgd(L.rowptr, L.rowind, L.rowval, b, err, k, threads=cores)
    t0 = time.perf_counter()
    run(10)
    t_iter = (time.perf_counter() - t0) / 10
    block = int(max(20, min(ref_it, 1.5 / max(t_iter, 1e-9))))
    step_s = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        _, done, _ = run(block)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            step_s.append(dt / max(done, 1) * block)
    s_block = float(np.median(step_s))
    v = 1.0 / (s_block / block * ref_it)
    info = {"kind": kind, "cores": cores, "iterations_timed": block}
    return {
        "impl": "reference",
        "metric": "CG solves/s (FP64, 2D 5-point Laplacian 1024x1024, rel-res 1e-8)",
        "value": v, "unit": "solves/s", "n_gpus": args.gpus, "gpus_used": 0,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * s_block, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded b ~ U[-1,1] (seed 2), exact 5-point Laplacian",
        "config": {"workload": "cg_laplace2d_1024 (plain FP64 CG, x0=0, rel-res 1e-8, max 5000 it)",
                   "n": L.nrows, "nnz": L.nnz, "reference_iterations": ref_it,
                   "step": (f"one timed block of {block} of the {ref_it} iterations of a "
                            "fresh solve; ms_per_step is that block's time"),
                   "omp": {"threads": cores, "OMP_PROC_BIND": os.environ.get("OMP_PROC_BIND"),
                           "OMP_PLACES": os.environ.get("OMP_PLACES"),
                           "logical_cpus": os.cpu_count()}},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": info["cores"],
                         "kind": info["kind"],
                         "sample": (f"per step {info['iterations_timed']} of {ref_it} "
                                    "iterations of the reference cgd, scaled to a full solve")},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="cg_laplace2d")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the secondary workloads reported under 'extras'")
    ap.add_argument("--requests", type=int, default=300,
                    help="requests of the serving stream (extras / --workload serving)")
    args = ap.parse_args()
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)

    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        pin_openmp()
        out = run_reference_cg(args)
        print(json.dumps(out), flush=True)
        return 0

    dist = Dist()
    try:
        if args.workload == "cg_laplace2d":
            out = run_cg_laplace(args, dist)
            if dist.world == 1 and not args.no_extras:
                out["extras"] = run_extras(args)
        elif args.workload in ("spmv_uniform", "spmv_powerlaw"):
            out = run_spmv(args, dist, args.workload)
        elif args.workload == "cg_mixed_3d":
            out = {"extras": {"mixed_cg_3d_160": mixed_extra(peak=hbm_peak()[0])}}
        elif args.workload == "serving":
            out = {"extras": {"serving_stream": serving_extra(nreq=args.requests)}}
        elif args.workload == "spmm":
            out = {"extras": {"spmm_laplace1024_k8": spmm_extra(peak=hbm_peak()[0])}}
        elif args.workload == "loader":
            out = {"extras": {"csr_loader_2m": loader_extra()}}
        elif args.workload == "pagerank":
            out = {"extras": {"pagerank_powerlaw_2m": pagerank_extra()}}
        elif args.workload == "rcm":
            import torch
            flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
            from gooseberry_b200 import workloads as W
            A = W.powerlaw_rows(8_000_000, 128_000_000, seed=3, cap=200_000)
            out = {"extras": {"rcm_reorder": rcm_extra(A, flush)}}
        else:
            raise SystemExit(f"unknown workload {args.workload}")
        if dist.rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
