#!/usr/bin/env python
"""Benchmark of the Merbit merge-path CSR SpMV on B200.

Workload (default): the power-law matrix -- 2,000,000 x 2,000,000, row
lengths Zipf(1.8) capped at 200,000, 10% empty rows, sorted unique uniform
columns, values N(0,1), x ~ U[-1,1], seed 1 -- in plain FP64 (values, x, y
and accumulation).  It stands in for the reference harness's Matrix Market
graphs, which are not available; the generator is merbit_b200/synth.py.

One step = one SpMV  y = A x  over the resident matrix (the reference's
harness times the same unit: tim2 / 400, include/tile.cuh:599-608).

  value  GB/s of algorithmic traffic, B = 4(nrow+1) + nnz(4+8) + 8 ncol + 8 nrow,
         over K back-to-back steps timed with CUDA events on the launching
         stream; the matrix (~0.6 GB) is larger than L2, so each step streams
         it from HBM (x, 16 MB, may stay in L2 between steps).
  e2e    the same metric through the public API (merbit_b200.Plan.spmv) with
         host buffers: every step copies x from pinned host memory, runs the
         SpMV and copies y back; consecutive steps are pipelined over three
         streams (the copies of steps i+1 and i-1 overlap step i's SpMV).
  roofline  the SpMV kernel's algorithmic bytes / its mean launch time vs the
         measured HBM copy bandwidth (MEASURED_PEAKS.json).
  cpu_baseline  the merge-path OpenMP FP64 SpMV of the CPU oracle on all host
         cores (the reference ships no CPU SpMV; this is its restatement).

Multi-GPU (torchrun): each rank runs its own copy of the workload (weak
scaling, no data-path collective); value = all ranks' bytes / the slowest
rank's time.

--impl reference times the CPU restatement on this host's cores as the
reference arm, and the reference's own merbit_kernel (built from the
reference sources into oracle/_ref) on the GPU as an extra field.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "SpMV GB/s (% of HBM peak) & GFLOP/s; mixed/batched vs plain FP64 at 1e-6 rel"
FALLBACK_HBM_GBS = 6650.0
KERNEL_OF_KIND = {0: "spmv_tile_kernel", 1: "spmv_warp_kernel", 3: "spmv_rows_kernel"}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="zipf_2m")
    ap.add_argument("--dtype", choices=["f64", "f32", "bf16"], default="f64")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--config", type=int, default=-1,
                    help="force SpMV kernel configuration index (skips tuning)")
    ap.add_argument("--k", type=int, default=8,
                    help="right-hand sides of the batched form (--workload rmat_batch128)")
    ap.add_argument("--batch", type=int, default=128, help="matrices of the batched form")
    ap.add_argument("--batch-tile", type=int, default=0,
                    help="batched form: run the SpMM kernel with this many merge items per "
                         "tile for every matrix (merbit_batch_set_kernel) instead of the "
                         "default or tuned choice")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the secondary forms (stencil precision form, batched form, "
                         "differentiation form) that the default power-law run adds")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def alg_bytes(A, dtype: str, k: int = 1) -> float:
    sv = {"f64": 8, "f32": 4, "bf16": 2}[dtype]
    sxy = 8 if dtype == "f64" else 4
    return 4.0 * (A.nrow + 1) + A.nnz * (4.0 + sv) + k * sxy * (A.ncol + A.nrow)


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
        0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
        0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
        0x100: "display_clock_setting",
    }

    def __init__(self, index: int, period_s: float = 0.005):
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._ok = False
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._ok = True
        except Exception:
            self._ok = False
        self.period = period_s
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                self.samples.append((mhz, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def start(self):
        if self._ok:
            self._t.start()
        return self

    def stop(self):
        self._stop.set()
        if self._ok:
            self._t.join()
        return self

    def summary(self):
        if not self._ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml_unavailable"],
                    "samples": 0}
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        mhz = [m for m, _ in self.samples]
        bits = 0
        for _, r in self.samples:
            bits |= r
        reasons = [n for b, n in self.REASONS.items() if bits & b and n != "gpu_idle"]
        return {"sm_mhz": float(statistics.median(mhz)), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(mhz)}


def dist_env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def dist_setup(args, backend: str | None = None, timeout_s: float = 120.0):
    """One process per GPU: the process group (NCCL on GPUs, gloo otherwise)
    with a short timeout, and this rank's device."""
    import torch

    ws, rank, local = dist_env()
    cuda = torch.cuda.is_available()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        backend = backend or ("nccl" if cuda else "gloo")
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    elif cuda:
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def allreduce_max(ws, v: float) -> float:
    """The maximum of v over ranks (every rank gets it)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_value(ws: int, units_per_rank: float, ms_max: float) -> float:
    """Whole-job throughput of a weak-scaling run: every rank processed
    units_per_rank; the job took as long as its slowest rank."""
    return ws * units_per_rank / (ms_max * 1e-3)


def load(args):
    from merbit_b200 import synth

    A = synth.workload(args.workload)
    x = synth.workload_x(args.workload, A.ncol)
    return A, x


L2_BYTES = 126 * 1024 * 1024


def l2_note(A, dtype: str) -> str:
    if alg_bytes(A, dtype) > L2_BYTES:
        return ("inputs larger than L2 (the matrix is streamed from HBM every step); "
                "value_l2_flushed flushes L2 before every launch")
    return ("matrix fits in L2 (L2-resident between back-to-back steps); "
            "value_l2_flushed flushes L2 before every launch")


def workload_config(args, A) -> dict:
    """The workload both arms print, as one identical dict."""
    return {"workload": args.workload, "nrow": A.nrow, "ncol": A.ncol, "nnz": A.nnz,
            "values": args.dtype, "k": 1, "l2": l2_note(A, args.dtype)}


def cpu_baseline(A, x, seconds: float):
    """Timed OpenMP FP64 merge-path SpMV (oracle/, CPU restatement)."""
    from oracle import oracle as O

    y = np.empty(A.nrow)
    vals = np.ascontiguousarray(A.vals, np.float64)
    O.spmv_omp_f64(A.row_ptr, A.col, vals, x, y)  # warm-up (page-in, thread spin-up)
    times = []
    t_end = time.perf_counter() + seconds
    threads = 1
    while time.perf_counter() < t_end or len(times) < 3:
        t0 = time.perf_counter()
        _, threads = O.spmv_omp_f64(A.row_ptr, A.col, vals, x, y)
        times.append(time.perf_counter() - t0)
        if len(times) >= 200:
            break
    med = statistics.median(times)
    return y, med, threads, len(times)


def gather_ceiling(A, dev, stream, reps: int = 10):
    """Random-gather rate of this GPU (G gathers/s): a pure gather loop over
    nnz uniformly random columns of a double vector of ncol entries."""
    import ctypes as C

    import torch

    import merbit_b200 as mb

    n = A.nnz - A.nnz % 16
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    idx = torch.randint(0, A.ncol, (n,), dtype=torch.int32, device=dev, generator=g)
    xg = torch.rand(A.ncol, dtype=torch.float64, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    out = torch.empty(sms * 2048, dtype=torch.float64, device=dev)
    L = mb.lib()
    sp = C.c_void_p(stream.cuda_stream)

    def launch():
        mb._check(L.merbit_bench_gather(C.c_void_p(xg.data_ptr()), A.ncol,
                                        C.c_void_p(idx.data_ptr()), n,
                                        C.c_void_p(out.data_ptr()), out.numel(), sp))

    for _ in range(3):
        launch()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        launch()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    sec = e0.elapsed_time(e1) / reps * 1e-3
    del idx, xg, out
    return n / sec / 1e9


def traffic_from_profile(workload: str, dtype: str):
    p = os.path.join(ROOT, "profiles", f"spmv_{dtype}_{workload}_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


def fast_tiles(rp, A, info) -> dict:
    """Tiles that end no row -- the single-row path (the reference's
    fast_track, include/tile.cuh:267-290; counted by its tile_desc_kernel,
    include/tile.cuh:178-210).  For the reference plan format (32 lanes x 14
    items, the fast flag in tile_y's MSB) and for the partition of the
    kernel in use (its nr == 0 tiles), the fraction of tiles and of
    nonzeros on that path."""
    import torch

    import merbit_b200 as mb

    out = {}
    tx, ty, _ = mb.tile_build(rp, A.nnz, 14)
    t = ty.numel() - 1
    fast = (ty[:-1].view(torch.int32) < 0)  # MSB set
    nz = (tx[1:] - tx[:-1]).to(torch.int64)
    out["reference_plan_sigma14"] = {
        "tiles": int(t), "fast_tiles": int(fast.sum()),
        "frac_tiles": round(float(fast.sum()) / max(t, 1), 4),
        "frac_nnz": round(float(nz[fast].sum()) / max(A.nnz, 1), 4)}
    if info.kind in (0, 1) and info.num_tiles > 0:
        T = info.num_tiles
        cx, cy = mb.merge_coords(rp, A.nnz, info.tile_items, T + 1)
        f = cy[1:] == cy[:-1]
        n = (cx[1:] - cx[:-1]).to(torch.int64)
        out["kernel_partition"] = {
            "tile_items": info.tile_items, "tiles": int(T), "single_row_tiles": int(f.sum()),
            "frac_tiles": round(float(f.sum()) / T, 4),
            "frac_nnz": round(float(n[f].sum()) / max(A.nnz, 1), 4)}
    else:
        out["kernel_partition"] = None  # row-group kernel: no merge-path tiles
    return out


def graph_time(launch, steps: int, dev, stream, local: int = 0):
    """Mean device time (ms) of one launch(stream) call: `steps` calls are
    captured into one CUDA graph, replayed once untimed (upload) and once
    inside CUDA events; NVML clocks are sampled meanwhile."""
    import torch

    g = torch.cuda.CUDAGraph()
    cap = torch.cuda.Stream(dev)
    cap.wait_stream(stream)
    with torch.cuda.graph(g, stream=cap):
        for _ in range(steps):
            launch(cap)
    stream.wait_stream(cap)
    g.replay()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local).start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.replay()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    sampler.stop()
    del g
    return e0.elapsed_time(e1) / steps, sampler.summary()


def component_error(y, y_ref, y_abs) -> dict:
    """max and median of |y - y_ref| / max(sum_j |a_ij x_j|, tiny)."""
    e = np.abs(np.asarray(y, np.float64) - y_ref) / np.maximum(y_abs, 1e-300)
    if e.size == 0:
        return {"max": 0.0, "median": 0.0}
    return {"max": float(e.max()), "median": float(np.median(e))}


def l2_flushed_ms(A, rp, col, vals64, x64, dev, stream, reps: int = 20) -> float:
    """Mean ms of one tuned FP64 SpMV launched after writing a 256 MB buffer
    (larger than L2), each launch timed on its own with CUDA events."""
    import torch

    import merbit_b200 as mb

    plan = mb.Plan(rp, col, vals64, ncol=A.ncol)
    plan.tune(x64)
    y = torch.empty(A.nrow, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(reps)]
    for a, b in evs:
        flush.fill_(1)
        a.record(stream)
        plan.spmv(x64, y)
        b.record(stream)
    torch.cuda.synchronize(dev)
    plan.close()
    return statistics.mean(a.elapsed_time(b) for a, b in evs)


def cpu_fp64_error(A, vals_stored, x_stored, y_gpu) -> dict:
    """Component-wise error of y_gpu against the FP64 CPU SpMV (the OpenMP
    restatement of the CPU baseline, oracle/) on the inputs as stored."""
    from oracle import oracle as O

    ys, _ = O.spmv_omp_f64(A.row_ptr, A.col, vals_stored, x_stored)
    ya = O.spmv_abs_omp_f64(A.row_ptr, A.col, vals_stored, x_stored)
    return component_error(y_gpu, ys, ya)


def spmv_form(A, dtype: str, rp, col, vals64, x64, steps: int, dev, stream, peak: float,
              workload: str, cpu_check: bool = True) -> dict:
    """One tuned SpMV of A with values stored as `dtype` (x FP64 for FP64
    values, FP32 otherwise), timed over `steps` graph-captured launches, with
    its error against an FP64 SpMV (the OpenMP oracle) of the inputs as
    stored."""
    import torch

    import merbit_b200 as mb
    vt = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16}[dtype]
    xt = torch.float64 if dtype == "f64" else torch.float32
    vals = vals64.to(vt)
    x = x64.to(xt)
    y = torch.empty(A.nrow, dtype=xt, device=dev)
    plan = mb.Plan(rp, col, vals, ncol=A.ncol)
    plan.tune(x)
    info = plan.info()
    for _ in range(3):
        plan.spmv(x, y)
    ms, clk = graph_time(lambda s: plan.spmv(x, y, stream=s), steps, dev, stream)
    plan.check()
    B = alg_bytes(A, dtype)
    gbs = B / (ms * 1e-3) / 1e9
    y_gpu = y.cpu().numpy()
    out = {
        "ms": round(ms, 5), "gbs": round(gbs, 2), "gflops": round(2.0 * A.nnz / (ms * 1e-3) / 1e9, 2),
        "algorithmic_bytes": B,
        "roofline": {"bound": "hbm", "achieved": round(gbs, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(gbs / peak, 4),
                     "traffic": traffic_from_profile(workload, dtype),
                     "kernel": KERNEL_OF_KIND[info.kind]},
        "kernel": f"{KERNEL_OF_KIND[info.kind]} block={info.block} ipt={info.items_per_thread} "
                  f"tile_items={info.tile_items} l1_carveout={info.l1_carveout} "
                  f"gather_l2_only={int(info.gather_l2_only)}",
        "clocks": clk,
    }
    if cpu_check:
        # CPU-baseline leg: the FP64 CPU SpMV (OpenMP restatement) of the
        # values and x as stored, against which the error is taken
        out["err_vs_fp64_stored_inputs"] = cpu_fp64_error(
            A, vals.to(torch.float64).cpu().numpy(), x.to(torch.float64).cpu().numpy(), y_gpu)
    plan.close()
    return out


def batch_forms(steps: int, dev, stream, peak: float, count: int = 128, ks=(1, 32)) -> dict:
    """The batched form against the plain form on the same matrices at the
    same k: `count` R-MAT matrices (seed 2) with FP32 values in one
    persistent, graph-captured, tuned launch, against one plain FP64 launch
    per matrix (tuned SpMV at k = 1, SpMM otherwise), also graph-captured."""
    import torch

    import merbit_b200 as mb
    from merbit_b200 import synth

    t0 = time.perf_counter()
    specs = synth.batch_rmat_specs(count, seed=2)
    mats = [synth.rmat(n, d, seed=sd) for n, d, sd in specs]
    t_gen = time.perf_counter() - t0
    nnz = sum(A.nnz for A in mats)
    dev_mats = []
    for A in mats:
        rp = torch.from_numpy(A.row_ptr).to(dev)
        col = torch.from_numpy(np.ascontiguousarray(A.col)).to(dev)
        v64 = torch.from_numpy(np.ascontiguousarray(A.vals)).to(dev)
        dev_mats.append((rp, col, v64))
    out = {"matrices": count, "nnz": nnz, "rows": sum(A.nrow for A in mats),
           "generate_s": round(t_gen, 2)}
    for k in ks:
        Xh = [synth.uniform(100 + i, A.ncol * k).astype(np.float32).reshape(A.ncol, k)
              for i, A in enumerate(mats)]
        # batched form: FP32 values, one launch
        p32, X32, Y32 = [], [], []
        for (rp, col, v64), A, X in zip(dev_mats, mats, Xh):
            p32.append(mb.Plan(rp, col, v64.to(torch.float32), ncol=A.ncol))
            X32.append(torch.from_numpy(X).to(dev))
            Y32.append(torch.empty(A.nrow, k, dtype=torch.float32, device=dev))
        batch = mb.Batch(p32, X32, Y32)
        batch.tune()
        binfo = batch.info()
        per_matrix = {}
        for kern, tile, ipt in batch.matrix_configs():
            per_matrix[tile] = per_matrix.get(tile, 0) + 1
        bkernel = (f"batch_warp_kernel variant {binfo['variant']}" if binfo["kernel"] == 1 else
                   f"spmm_kernel vector_width={binfo['vector_width']}")
        batch.run()
        ms_b, clk_b = graph_time(lambda s: batch.run(stream=s), steps, dev, stream)
        # plain form: FP64 values, x and accumulation, one launch per matrix
        p64, X64, Y64 = [], [], []
        for (rp, col, v64), A, X in zip(dev_mats, mats, X32):
            p = mb.Plan(rp, col, v64, ncol=A.ncol)
            x64 = X.to(torch.float64)
            if k == 1:
                x64 = x64[:, 0].contiguous()
                p.tune(x64)
                Y64.append(torch.empty(A.nrow, dtype=torch.float64, device=dev))
            else:
                Y64.append(torch.empty(A.nrow, k, dtype=torch.float64, device=dev))
            p64.append(p)
            X64.append(x64)

        def plain(s):
            for p, x, y in zip(p64, X64, Y64):
                if k == 1:
                    p.spmv(x, y, stream=s)
                else:
                    p.spmm(x, y, stream=s)

        plain(stream)
        ms_p, clk_p = graph_time(plain, steps, dev, stream)
        # error of the batched FP32 result against the plain FP64 one, whose
        # denominators sum |a x| come from the same FP64 kernels on |A|, |X|
        torch.cuda.synchronize(dev)
        worst, meds = 0.0, []
        for (rp, col, v64), A, p, x, y64, y32 in zip(dev_mats, mats, p64, X64, Y64, Y32):
            pa = mb.Plan(rp, col, v64.abs(), ncol=A.ncol)
            ya = pa.spmv(x.abs()) if k == 1 else pa.spmm(x.abs())
            e = ((y32.reshape(y64.shape).double() - y64).abs() /
                 ya.clamp_min(1e-300)).flatten()
            if e.numel():
                worst = max(worst, float(e.max()))
                meds.append(float(e.median()))
            pa.close()
        b64 = sum(alg_bytes(A, "f64", k) for A in mats)
        b32 = binfo["algorithmic_bytes"]
        out[f"k{k}"] = {
            "batched_f32": {
                "ms": round(ms_b, 4), "gflops": round(2.0 * nnz * k / (ms_b * 1e-3) / 1e9, 2),
                "gbs": round(b32 / (ms_b * 1e-3) / 1e9, 2),
                "roofline": {"bound": "hbm", "achieved": round(b32 / (ms_b * 1e-3) / 1e9, 2),
                             "peak": peak, "unit": "GB/s",
                             "frac": round(b32 / (ms_b * 1e-3) / 1e9 / peak, 4),
                             "traffic": batch_traffic(k),
                             "kernel": bkernel.split()[0]},
                "launches_per_step": 1, "kernel": bkernel,
                "matrices_per_tile_items": {str(t): n for t, n in sorted(per_matrix.items())},
                "vector_width": binfo["vector_width"], "clocks": clk_b,
                "err_vs_plain_fp64": {"max": worst, "median": float(np.median(meds))},
            },
            "plain_f64": {
                "ms": round(ms_p, 4), "gflops": round(2.0 * nnz * k / (ms_p * 1e-3) / 1e9, 2),
                "gbs": round(b64 / (ms_p * 1e-3) / 1e9, 2), "launches_per_step": count,
                "clocks": clk_p,
                "kernel": "tuned SpMV per matrix" if k == 1 else "merge-path SpMM per matrix",
            },
        }
        batch.close()
        for p in p32 + p64:
            p.close()
        del X32, Y32, X64, Y64, Xh
    return out


def batch_traffic(k: int):
    p = os.path.join(ROOT, "profiles", f"batch_f32_rmat128_k{k}_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get("dram_bytes_per_launch")
    return None


def diff_measure(A, k: int, steps: int, dev, stream) -> dict:
    """Differentiation form: forward Y = A X and forward + backward (dX =
    A^T G and dval from one fused launch where the operands allow), FP32
    values, k right-hand sides; mean ms over `steps` back-to-back steps."""
    import torch

    from merbit_b200 import synth
    from merbit_b200.autograd import SparseMatrix

    rp = torch.from_numpy(A.row_ptr).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    vals = torch.from_numpy(A.vals.astype(np.float32)).to(dev)
    M = SparseMatrix(rp, col, vals, ncol=A.ncol)
    X = torch.from_numpy(synth.workload_x("zipf_1m_diff", A.ncol, k).astype(np.float32)).to(dev)
    G = torch.from_numpy(synth.normal(3, A.nrow * k).astype(np.float32).reshape(A.nrow, k)).to(dev)
    T = M.transpose_plan()
    Y = torch.empty(A.nrow, k, dtype=torch.float32, device=dev)
    dX = torch.empty(A.ncol, k, dtype=torch.float32, device=dev)

    def fwd():
        M.plan.spmm(X, Y)

    fused = M.backward_fused(G, X) is not None

    def bwd():
        if not fused or M.backward_fused(G, X) is None:
            T.spmm(G, dX)
            M.dval(G, X)

    for _ in range(3):
        fwd()
        bwd()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(0).start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fwd()
    e1.record(stream)
    for _ in range(steps):
        fwd()
        bwd()
    e2.record(stream)
    torch.cuda.synchronize(dev)
    sampler.stop()
    M.plan.check()
    t_f = e0.elapsed_time(e1) / steps
    t_fb = e1.elapsed_time(e2) / steps
    return {"fwd_ms": round(t_f, 4), "fwd_bwd_ms": round(t_fb, 4),
            "fwd_bwd_over_fwd": round(t_fb / t_f, 3),
            "backward": "fused transpose SpMM + dval (merbit_spmm_dval)" if fused
                        else "transpose SpMM, then dval",
            "launches_per_step": 2 if fused else 3, "fused": fused, "clocks": sampler.summary()}


def secondary_forms(args, A_zipf, rp, col, vals64, x64, dev, stream, peak,
                    ms_headline: float) -> tuple[dict, dict]:
    """The precision, batched and differentiation forms of the default run,
    each on its own benchmark matrix, plus the like-for-like ratios of the
    mixed or batched forms over the plain FP64 form."""
    import torch

    from merbit_b200 import synth

    # launches per measurement: up to 200 (one graph each); the batched
    # form's plain FP64 side is 128 launches per step, so it takes up to 50
    steps = min(args.steps, 200)
    batch_steps = min(args.steps, 50)
    forms, ratios = {"steps_per_measurement": steps,
                     "steps_per_measurement_batched": batch_steps}, {}
    t0 = time.perf_counter()
    # precision form on the power-law matrix itself (same matrix, same k = 1)
    chk = not args.no_cpu_baseline
    zf = {d: spmv_form(A_zipf, d, rp, col, vals64, x64, steps, dev, stream, peak, "zipf_2m", chk)
          for d in ("f32", "bf16")}
    forms["zipf_2m"] = zf
    # 5-point Laplacian 256^2, FP64 (L2-resident: 5.2 MB): back to back from
    # a graph, and one launch at a time with L2 flushed before each
    Lp = synth.workload("laplace2d_256")
    lrp = torch.from_numpy(Lp.row_ptr).to(dev)
    lcol = torch.from_numpy(Lp.col).to(dev)
    lv = torch.from_numpy(Lp.vals).to(dev)
    lx = torch.from_numpy(synth.workload_x("laplace2d_256", Lp.ncol)).to(dev)
    lap = spmv_form(Lp, "f64", lrp, lcol, lv, lx, steps, dev, stream, peak, "laplace2d_256", chk)
    lap["l2"] = "L2-resident between back-to-back launches (ms, gbs); ms_l2_flushed flushes L2"
    lap["ms_l2_flushed"] = round(l2_flushed_ms(Lp, lrp, lcol, lv, lx, dev, stream), 5)
    forms["laplace2d_256"] = {"nrow": Lp.nrow, "nnz": Lp.nnz, "f64": lap}
    del lrp, lcol, lv, lx, Lp
    # 27-point stencil 160^3 in FP64, FP32 and BF16
    S = synth.workload("stencil27_160")
    srp = torch.from_numpy(S.row_ptr).to(dev)
    scol = torch.from_numpy(S.col).to(dev)
    sv = torch.from_numpy(S.vals).to(dev)
    sx = torch.from_numpy(synth.workload_x("stencil27_160", S.ncol)).to(dev)
    st = {d: spmv_form(S, d, srp, scol, sv, sx, steps, dev, stream, peak, "stencil27_160", chk)
          for d in ("f64", "f32", "bf16")}
    forms["stencil27_160"] = {"nrow": S.nrow, "nnz": S.nnz, **st}
    del srp, scol, sv, sx, S
    torch.cuda.empty_cache()
    # batched form, k = 1 and 32
    bf = batch_forms(batch_steps, dev, stream, peak)
    forms["rmat_batch128"] = bf
    torch.cuda.empty_cache()
    # differentiation form: Zipf(1.8) 1M rows, k = 16
    D = synth.workload("zipf_1m_diff")
    forms["zipf_1m_diff_k16"] = {"nrow": D.nrow, "nnz": D.nnz,
                                 **diff_measure(D, 16, steps, dev, stream)}
    del D
    torch.cuda.empty_cache()
    forms["wall_s"] = round(time.perf_counter() - t0, 1)

    def ratio(plain_ms, mixed_ms, err, what):
        # err is None when the CPU-baseline leg (and its FP64 check) is off
        return {"speedup": round(plain_ms / mixed_ms, 3), "plain_f64_ms": plain_ms,
                "mixed_ms": mixed_ms, "err_max": err["max"] if err else None,
                "err_median": err["median"] if err else None,
                "within_1e-6": bool(err["max"] <= 1e-6) if err else None, "compares": what}

    for d in ("f32", "bf16"):
        ratios[f"zipf_2m_{d}_vs_f64"] = ratio(
            ms_headline, zf[d]["ms"], zf[d].get("err_vs_fp64_stored_inputs"),
            f"power-law 2M, k = 1: {d} values + f32 x vs plain FP64, same matrix")
        ratios[f"stencil27_160_{d}_vs_f64"] = ratio(
            st["f64"]["ms"], st[d]["ms"], st[d].get("err_vs_fp64_stored_inputs"),
            f"27-point stencil 160^3, k = 1: {d} values + f32 x vs plain FP64, same matrix")
    for k in (1, 32):
        b = bf[f"k{k}"]
        ratios[f"rmat_batch128_k{k}_batched_f32_vs_f64"] = ratio(
            b["plain_f64"]["ms"], b["batched_f32"]["ms"], b["batched_f32"]["err_vs_plain_fp64"],
            f"128 R-MAT matrices, k = {k}: one batched FP32 launch vs one plain FP64 launch "
            "per matrix, same matrices and right-hand sides")
    return forms, ratios


def run_ours(args):
    import torch

    import merbit_b200 as mb

    ws, rank, local = dist_setup(args)
    A, x = load(args)
    dev = torch.device("cuda", local)
    vt = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16}[args.dtype]
    xt = torch.float64 if args.dtype == "f64" else torch.float32
    rp = torch.from_numpy(A.row_ptr).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    vals = torch.from_numpy(A.vals).to(dev).to(vt)
    xd = torch.from_numpy(x).to(dev).to(xt)
    yd = torch.empty(A.nrow, dtype=xt, device=dev)
    torch.cuda.synchronize(dev)
    # loading the library (dlopen, its static CUDA runtime, registration of
    # its kernel images) is a once-per-process cost, timed on its own
    t_lib0 = time.perf_counter()
    mb.lib()
    t_lib = time.perf_counter() - t_lib0
    # plan build, as the reference's tim1 times its TILE build
    # (include/tile.cuh:587-593): CUDA events on the stream around it, and
    # the host wall time (allocation and synchronization included)
    ev_p0 = torch.cuda.Event(enable_timing=True)
    ev_p1 = torch.cuda.Event(enable_timing=True)
    ev_p0.record(torch.cuda.current_stream(dev))
    t_plan0 = time.perf_counter()
    plan = mb.Plan(rp, col, vals, ncol=A.ncol)  # validates, partitions; synchronizes
    t_plan = time.perf_counter() - t_plan0
    ev_p1.record(torch.cuda.current_stream(dev))
    torch.cuda.synchronize(dev)
    t_plan_ev = ev_p0.elapsed_time(ev_p1)
    # the first build in a process also pays the one-time CUDA module load
    # of the library; later builds of a plan (median of 5) do not
    warm = []
    for _ in range(5):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        q = mb.Plan(rp, col, vals, ncol=A.ncol)
        warm.append(time.perf_counter() - t0)
        q.close()
    t_plan_warm = statistics.median(warm)
    if args.config >= 0:
        plan.set_config(args.config)
    elif not args.no_tune:
        plan.tune(xd)
    info = plan.info()
    B = alg_bytes(A, args.dtype)
    stream = torch.cuda.current_stream(dev)

    for _ in range(max(args.warmup, 3)):
        plan.spmv(xd, yd)
    torch.cuda.synchronize(dev)

    # ---- timed region: K back-to-back steps, captured once as a CUDA graph
    # (merbit_spmv neither allocates nor synchronizes) so that per-call host
    # work stays out of the device timing of small, launch-bound matrices
    graph = torch.cuda.CUDAGraph()
    cap = torch.cuda.Stream(dev)
    cap.wait_stream(stream)
    with torch.cuda.graph(graph, stream=cap):
        for _ in range(args.steps):
            plan.spmv(xd, yd, stream=cap)
    stream.wait_stream(cap)
    graph.replay()  # untimed: the graph's first launch uploads it
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local).start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    graph.replay()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    sampler.stop()
    del graph
    ms_local = e0.elapsed_time(e1) / args.steps
    ms = allreduce_max(ws, ms_local)
    plan.check()

    # ---- per-launch duration of the SpMV kernel with L2 flushed before each
    # launch (cold x as well as cold matrix)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    nflush = min(args.steps, 50)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(nflush)]
    for a, b in evs:
        flush.fill_(1)
        a.record(stream)
        plan.spmv(xd, yd)
        b.record(stream)
    torch.cuda.synchronize(dev)
    ms_cold = allreduce_max(ws, statistics.mean(a.elapsed_time(b) for a, b in evs))
    del flush

    # ---- the GPU's random-gather ceiling (merbit_bench_gather): nnz gathers
    # at uniformly random columns of a double x, 16 in flight per thread
    # (only for matrices with random columns, where it binds)
    gather = gather_ceiling(A, dev, stream) if args.workload.startswith("zipf") else None

    # ---- e2e through the public API with host buffers: every step copies
    # its x from pinned host memory, runs Plan.spmv and copies y back.  Steps
    # are pipelined over three streams (double-buffered device x and y): the
    # H2D copy of step i+1 and the D2H copy of step i-1 overlap the SpMV of
    # step i, as a serving loop would run them.
    xh = [torch.from_numpy(x).to(xt).pin_memory() for _ in range(2)]
    yh = [torch.empty(A.nrow, dtype=xt).pin_memory() for _ in range(2)]
    xdb = [torch.empty_like(xd) for _ in range(2)]
    ydb = [torch.empty_like(yd) for _ in range(2)]
    s_in = torch.cuda.Stream(dev)
    s_out = torch.cuda.Stream(dev)

    def e2e_steps(n):
        ev_c = [None, None]
        ev_out = [None, None]
        for i in range(n):
            b = i % 2
            if ev_c[b] is not None:
                s_in.wait_event(ev_c[b])  # step i-2's SpMV has read xdb[b]
            with torch.cuda.stream(s_in):
                xdb[b].copy_(xh[b], non_blocking=True)
            ev_in = torch.cuda.Event()
            ev_in.record(s_in)
            stream.wait_event(ev_in)
            if ev_out[b] is not None:
                stream.wait_event(ev_out[b])  # step i-2's D2H has read ydb[b]
            plan.spmv(xdb[b], ydb[b], stream=stream)
            ev_c[b] = torch.cuda.Event()
            ev_c[b].record(stream)
            s_out.wait_event(ev_c[b])
            with torch.cuda.stream(s_out):
                yh[b].copy_(ydb[b], non_blocking=True)
            ev_out[b] = torch.cuda.Event()
            ev_out[b].record(s_out)
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)

    ke = min(args.steps, 200)
    e2e_steps(4)
    barrier(ws)
    torch.cuda.synchronize(dev)
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    e2e_steps(ke)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(ws)
    ms_e2e = allreduce_max(ws, e0.elapsed_time(e1) / ke)
    y_gpu = yh[(ke - 1) % 2].numpy().astype(np.float64)

    if rank != 0:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    peak, peak_src = peaks()
    value = weak_value(ws, B, ms) / 1e9
    achieved = B / (ms * 1e-3) / 1e9
    traffic = traffic_from_profile(args.workload, args.dtype)
    out = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": round(ms, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": args.dtype,
        "data": "synthetic (seeded generator merbit_b200/synth.py; the reference's "
                "Matrix Market graphs are not available)",
        "config": workload_config(args, A),
        "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
        "launch": "the K timed SpMV launches captured in one CUDA graph, replayed once",
        "kernel": f"{KERNEL_OF_KIND[info.kind]} "
                  f"block={info.block} ipt={info.items_per_thread} "
                  f"tile_items={info.tile_items} tiles={info.num_tiles} "
                  f"vectorized={int(info.vectorized)} l1_carveout={info.l1_carveout} "
                  f"gather_l2_only={int(info.gather_l2_only)}",
        "fast_tiles": fast_tiles(rp, A, info),
        "pct_hbm_peak": round(100.0 * achieved / peak, 2),
        "gflops": round(ws * 2.0 * A.nnz / (ms * 1e-3) / 1e9, 2),
        "value_l2_flushed": round(ws * B / (ms_cold * 1e-3) / 1e9, 2),
        "algorithmic_bytes_per_step": B,
        "plan_metadata_bytes": info.metadata_bytes,
        "library_load_ms_host_wall": round(t_lib * 1e3, 3),
        "plan_build_ms_host_wall": round(t_plan * 1e3, 3),
        "plan_build_ms_events": round(t_plan_ev, 3),
        "plan_build_ms_warm_host_wall": round(t_plan_warm * 1e3, 3),
        "gpu_launches": args.steps,
        "roofline": {
            "bound": "hbm",
            "achieved": round(achieved, 2),
            "peak": peak,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "peak_source": f"{peak_src} hbm_gbs (copy), burst",
            "traffic": traffic,
            "kernel": KERNEL_OF_KIND[info.kind],
            "gather_bound": None if gather is None else {
                "achieved_ggather_s": round(A.nnz / (ms * 1e-3) / 1e9, 1),
                "ceiling_ggather_s": round(gather, 1),
                "frac": round(A.nnz / (ms * 1e-3) / 1e9 / gather, 4),
                "note": "one x gather per nonzero; ceiling = a pure random-gather loop on this "
                        "GPU (merbit_bench_gather). Binding when columns are random "
                        "(x misses L1), as for the power-law matrix",
            },
        },
        "e2e": {
            "value": round(ws * B / (ms_e2e * 1e-3) / 1e9, 2),
            "unit": "GB/s",
            "h2d_bytes_per_step": int(xh[0].numel() * xh[0].element_size()),
            "d2h_bytes_per_step": int(yh[0].numel() * yh[0].element_size()),
            "ms_per_step": round(ms_e2e, 5),
            "api": "merbit_b200.Plan.spmv (C ABI merbit_spmv)",
            "pipelining": "H2D of step i+1 and D2H of step i-1 overlap the SpMV of step i "
                          "(three streams, double-buffered device x and y)",
        },
        "clocks": sampler.summary(),
    }
    if ws == 1 and not args.no_forms and args.workload == "zipf_2m" and args.dtype == "f64":
        forms, ratios = secondary_forms(args, A, rp, col, vals, xd, dev, stream, peak, ms)
        out["forms"] = forms
        out["mixed_vs_plain"] = ratios
    if ws == 1 and not args.no_cpu_baseline:
        y_cpu, t_cpu, threads, reps = cpu_baseline(A, x, args.cpu_seconds)
        out["cpu_baseline"] = {
            "value": round(B / t_cpu / 1e9, 3),
            "unit": "GB/s",
            "cores": threads,
            "kind": "port",
            "sample": f"full {args.workload} matrix, FP64, median of {reps} SpMVs "
                      f"(merge-path OpenMP restatement in oracle/merbit_oracle.c)",
        }
        # component-wise error |y - y_cpu| / sum_j |a_ij x_j|
        rows = np.repeat(np.arange(A.nrow), np.diff(A.row_ptr))
        yabs = np.bincount(rows, weights=np.abs(A.vals) * np.abs(x[A.col]), minlength=A.nrow)
        rel = np.abs(y_gpu - y_cpu) / np.maximum(yabs, 1e-300)
        out["err_vs_cpu_fp64"] = {"max": float(rel.max()), "median": float(np.median(rel)),
                                  "note": "component-wise, vs the FP64 CPU baseline's y"}
        if args.dtype != "f64":
            # the kernel's own error: FP64 oracle on the inputs as stored
            # (values rounded to f32/bf16, x to f32)
            from oracle import oracle as O

            vt = {"f32": torch.float32, "bf16": torch.bfloat16}[args.dtype]
            vs = torch.from_numpy(np.ascontiguousarray(A.vals)).to(vt).to(torch.float64).numpy()
            xs = x.astype(np.float32).astype(np.float64)
            ys = np.empty(A.nrow)
            O.spmv_omp_f64(A.row_ptr, A.col, vs, xs, ys)
            ya = np.bincount(rows, weights=np.abs(vs) * np.abs(xs[A.col]), minlength=A.nrow)
            rs = np.abs(y_gpu - ys) / np.maximum(ya, 1e-300)
            out["err_vs_fp64_stored_inputs"] = {
                "max": float(rs.max()), "median": float(np.median(rs)),
                "note": "component-wise, vs an FP64 SpMV of the values and x as stored "
                        "(the accumulation error; err_vs_cpu_fp64 adds the input rounding)"}
    print(json.dumps(out), flush=True)


def load_batch(args):
    from merbit_b200 import synth

    specs = synth.batch_rmat_specs(args.batch, seed=2)
    mats = [synth.rmat(n, d, seed=sd) for n, d, sd in specs]
    xs = [synth.uniform(100 + i, A.ncol * args.k).astype(np.float32).reshape(A.ncol, args.k)
          for i, A in enumerate(mats)]
    return mats, xs


def run_batch(args):
    """Batched form: 128 R-MAT matrices (rows log-uniform in [1e3, 5e5], average
    degree uniform in [8, 64], FP32 values N(0,1)) times k FP32 right-hand
    sides, one graph-captured persistent launch per step."""
    import torch

    import merbit_b200 as mb

    ws, rank, local = dist_setup(args)
    dev = torch.device("cuda", local)
    mats, xs = load_batch(args)
    k = args.k
    plans, Xd, Yd = [], [], []
    for A, X in zip(mats, xs):
        rp = torch.from_numpy(A.row_ptr).to(dev)
        col = torch.from_numpy(A.col).to(dev)
        v = torch.from_numpy(A.vals.astype(np.float32)).to(dev)
        plans.append(mb.Plan(rp, col, v, ncol=A.ncol))
        Xd.append(torch.from_numpy(X).to(dev))
        Yd.append(torch.empty(A.nrow, k, dtype=torch.float32, device=dev))
    batch = mb.Batch(plans, Xd, Yd)
    if args.batch_tile:
        batch.set_kernel(0, args.batch_tile)
    elif not args.no_tune:
        batch.tune()
    info = batch.info()
    per_matrix = {}
    for _, tile, _ in batch.matrix_configs():
        per_matrix[str(tile)] = per_matrix.get(str(tile), 0) + 1
    kname = "batch_warp_kernel" if info["kernel"] == 1 else "spmm_kernel"
    stream = torch.cuda.Stream(dev)
    stream.wait_stream(torch.cuda.current_stream(dev))
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        batch.run(stream=stream)
    for _ in range(max(args.warmup, 3)):
        graph.replay()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local).start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_stream(dev)
    barrier(ws)
    torch.cuda.synchronize(dev)
    e0.record(cur)
    for _ in range(args.steps):
        graph.replay()
    e1.record(cur)
    torch.cuda.synchronize(dev)
    barrier(ws)
    sampler.stop()
    ms = allreduce_max(ws, e0.elapsed_time(e1) / args.steps)
    # e2e: X from pinned host memory, one replay, Y back, per step
    xh = [torch.from_numpy(X).pin_memory() for X in xs]
    yh = [torch.empty(A.nrow, k, dtype=torch.float32).pin_memory() for A in mats]
    ke = min(args.steps, 5)
    e0.record(cur)
    for _ in range(ke):
        for a, b in zip(Xd, xh):
            a.copy_(b, non_blocking=True)
        graph.replay()
        for a, b in zip(yh, Yd):
            a.copy_(b, non_blocking=True)
    e1.record(cur)
    torch.cuda.synchronize(dev)
    ms_e2e = allreduce_max(ws, e0.elapsed_time(e1) / ke)
    del graph
    if rank != 0:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    B = info["algorithmic_bytes"]
    peak, peak_src = peaks()
    achieved = B / (ms * 1e-3) / 1e9
    out = {
        "metric": METRIC,
        "value": round(ws * achieved, 2),
        "unit": "GB/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": round(ms, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded R-MAT generator, merbit_b200/synth.py)",
        "config": {"workload": f"rmat_batch{args.batch}", "matrices": len(mats), "k": k,
                   "nnz": int(info["nnz"]), "rows": int(sum(A.nrow for A in mats)),
                   "l2": "inputs larger than L2"},
        "launch": "one persistent kernel per step, CUDA-graph replay",
        "kernel": f"{kname} variant={info['variant']} vector_width={info['vector_width']}",
        "matrices_per_tile_items": per_matrix,
        "pct_hbm_peak": round(100.0 * achieved / peak, 2),
        "gflops": round(ws * 2.0 * info["nnz"] * k / (ms * 1e-3) / 1e9, 2),
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "peak_source": f"{peak_src} hbm_gbs (copy), burst",
                     "traffic": batch_traffic(k) if args.batch == 128 else None,
                     "kernel": kname},
        "e2e": {"value": round(ws * B / (ms_e2e * 1e-3) / 1e9, 2), "unit": "GB/s",
                "h2d_bytes_per_step": int(sum(X.nbytes for X in xs)),
                "d2h_bytes_per_step": int(sum(A.nrow * k * 4 for A in mats)),
                "ms_per_step": round(ms_e2e, 4),
                "api": "merbit_b200.Batch.run (C ABI merbit_batch_spmm), graph-captured"},
        "clocks": sampler.summary(),
    }
    if ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O

        t_cpu, b_cpu, threads, n_done = 0.0, 0.0, 1, 0
        worst, errs = 0.0, []
        for A, X, Y in zip(mats, xs, yh):
            v32 = A.vals.astype(np.float32)
            t0 = time.perf_counter()
            yc, threads = O.spmm_omp_f32(A.row_ptr, A.col, v32, X, k)
            t_cpu += time.perf_counter() - t0
            b_cpu += 4.0 * (A.nrow + 1) + A.nnz * 8.0 + 4.0 * k * (A.ncol + A.nrow)
            rows = np.repeat(np.arange(A.nrow), np.diff(A.row_ptr))
            den = np.zeros((A.nrow, k))
            np.add.at(den, rows, np.abs(v32.astype(np.float64))[:, None] *
                      np.abs(X[A.col].astype(np.float64)))
            e = np.abs(Y.numpy().astype(np.float64) - yc) / np.maximum(den, 1e-300)
            worst = max(worst, float(e.max()) if e.size else 0.0)
            errs.append(float(np.median(e)) if e.size else 0.0)
            n_done += 1
            if t_cpu > args.cpu_seconds:
                break
        out["cpu_baseline"] = {"value": round(b_cpu / t_cpu / 1e9, 3), "unit": "GB/s",
                               "cores": threads, "kind": "port",
                               "sample": f"first {n_done} of {len(mats)} matrices, one SpMM each "
                                         "(row-parallel OpenMP float SpMM, oracle/merbit_oracle.c)"}
        out["err_vs_cpu"] = {"max": worst, "median": float(np.median(errs)),
                             "note": "component-wise, vs the CPU baseline's double-accumulated Y, "
                                     "on the matrices the CPU sample covered"}
    print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_diff(args):
    """Differentiation form: Y = A X (k RHS, FP32 values) forward, and the
    backward dX = A^T G, dval = G[row].X[col], on the Zipf(1.8) 1M-row
    matrix (seed 3); reports forward and forward+backward times."""
    import torch

    from merbit_b200 import synth

    ws, rank, local = dist_setup(args)
    dev = torch.device("cuda", local)
    A = synth.workload(args.workload)
    k = args.k
    barrier(ws)
    d = diff_measure(A, k, args.steps, dev, torch.cuda.current_stream(dev))
    barrier(ws)
    t_f = allreduce_max(ws, d["fwd_ms"])
    t_fb = allreduce_max(ws, d["fwd_bwd_ms"])
    if rank != 0:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    B = 4.0 * (A.nrow + 1) + A.nnz * 8.0 + 4.0 * k * (A.ncol + A.nrow)
    peak, peak_src = peaks()
    out = {
        "metric": METRIC,
        "value": round(ws * B / (t_f * 1e-3) / 1e9, 2),
        "unit": "GB/s",
        "n_gpus": ws, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": round(t_f, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded Zipf(1.8) generator, merbit_b200/synth.py)",
        "config": {"workload": args.workload, "nrow": A.nrow, "ncol": A.ncol, "nnz": A.nnz,
                   "values": "f32", "k": k, "l2": "inputs larger than L2"},
        "fwd_ms": round(t_f, 4),
        "fwd_bwd_ms": round(t_fb, 4),
        "fwd_bwd_over_fwd": round(t_fb / t_f, 3),
        "gpu_launches": (1 + d["launches_per_step"]) * args.steps,
        "backward": d["backward"],
        "roofline": {"bound": "hbm", "achieved": round(B / (t_f * 1e-3) / 1e9, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(B / (t_f * 1e-3) / 1e9 / peak, 4),
                     "peak_source": f"{peak_src} hbm_gbs", "traffic": None,
                     "kernel": "spmm_kernel (forward)"},
        "clocks": d["clocks"],
    }
    print(json.dumps(out), flush=True)


def run_reference(args):
    """The reference arm: rank 0 alone times the CPU implementation; other
    ranks exit at once (no process group, nothing to wait for)."""
    import torch

    ws, rank, local = dist_env()
    if rank != 0:
        return
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    from oracle import oracle as O

    A, x = load(args)
    B = alg_bytes(A, "f64")
    vals = np.ascontiguousarray(A.vals, np.float64)
    y = np.empty(A.nrow)
    O.spmv_omp_f64(A.row_ptr, A.col, vals, x, y)
    per_step = []
    threads = 1
    # each step: one SpMV over the full matrix on all host cores; the run
    # stops after ~cpu_seconds even when more steps were requested
    for _ in range(max(args.warmup, 3)):
        O.spmv_omp_f64(A.row_ptr, A.col, vals, x, y)
    t_stop = time.perf_counter() + max(args.cpu_seconds, 5.0) * 3
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, threads = O.spmv_omp_f64(A.row_ptr, A.col, vals, x, y)
        per_step.append(time.perf_counter() - t0)
        if time.perf_counter() > t_stop:
            break
    sec = statistics.median(per_step)
    value = B / sec / 1e9
    out = {
        "metric": METRIC,
        "impl": "reference",
        "value": round(value, 3),
        "unit": "GB/s",
        "n_gpus": ws,
        "steps": len(per_step),
        "warmup": max(args.warmup, 3),
        "ms_per_step": round(sec * 1e3, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded generator merbit_b200/synth.py)",
        "config": workload_config(args, A),
        "cpu_baseline": {
            "value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"full {args.workload} matrix per step, median of {len(per_step)} steps; "
                      "the reference has no CPU SpMV, this is the merge-path OpenMP "
                      "restatement (oracle/merbit_oracle.c)",
        },
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    # the reference's own GPU kernel (merbit_kernel<double,256,14>, built from
    # the reference sources) on the same matrix, for comparison
    R = O.ref()
    if R is not None and torch.cuda.is_available():
        dev = torch.device("cuda", local)
        rp = torch.from_numpy(A.row_ptr).to(dev)
        col = torch.from_numpy(A.col).to(dev)
        v = torch.from_numpy(vals).to(dev)
        xd = torch.from_numpy(x).to(dev)
        yd = torch.zeros(A.nrow, dtype=torch.float64, device=dev)
        zd = torch.zeros(A.nrow, dtype=torch.float64, device=dev)
        lane_num = (A.nrow + A.nnz + 13) // 14
        tile_num = (lane_num + 31) // 32
        tx = torch.zeros(tile_num + 1, dtype=torch.int32, device=dev)
        ty = torch.zeros(tile_num + 1, dtype=torch.int32, device=dev)
        desc = torch.zeros(max(lane_num, 1), dtype=torch.int32, device=dev)
        t0 = time.perf_counter()
        rc = R.ref_tile_build(14, rp.data_ptr(), A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(),
                              desc.data_ptr())
        t_plan = time.perf_counter() - t0
        warm = []
        for _ in range(5):  # later builds, without the one-time module load
            t0 = time.perf_counter()
            R.ref_tile_build(14, rp.data_ptr(), A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(),
                             desc.data_ptr())
            warm.append(time.perf_counter() - t0)
        if rc == 0:
            s = torch.cuda.current_stream(dev).cuda_stream
            R.ref_merbit_time(0, col.data_ptr(), v.data_ptr(), A.nrow, A.nnz, tx.data_ptr(),
                              ty.data_ptr(), desc.data_ptr(), xd.data_ptr(), yd.data_ptr(),
                              zd.data_ptr(), 10, s)
            ms = R.ref_merbit_time(0, col.data_ptr(), v.data_ptr(), A.nrow, A.nnz,
                                   tx.data_ptr(), ty.data_ptr(), desc.data_ptr(), xd.data_ptr(),
                                   yd.data_ptr(), zd.data_ptr(), 400, s)
            out["ref_gpu_kernel"] = {
                "kernel": "merbit_kernel<double,256,14> (reference source, sm_100a build)",
                "value": round(B / (ms * 1e-3) / 1e9, 2), "unit": "GB/s",
                "ms_per_spmv": round(float(ms), 5), "reps": 400,
                "plan_build_s_host_wall": round(t_plan, 4),
                "plan_build_ms_warm_host_wall": round(statistics.median(warm) * 1e3, 3),
                "plan_build_note": "Tile_Kernel launch + device sync; its three arrays are "
                                   "allocated beforehand (torch), outside this time",
            }
        out["competitors_gpu"] = competitors(A, rp, col, v, xd, yd, zd, B, dev, y)
    print(json.dumps(out), flush=True)


def competitors(A, rp, col, v, xd, yd, zd, B, dev, y_cpu):
    """Run-only comparisons on the same FP64 matrix (GB/s of the same
    algorithmic bytes): the reference Merbit kernel with 64-bit lane
    descriptors (SIGMA 20), cuSPARSE through torch.sparse, and the libraries
    the reference's src/spmv.cu benchmarks (library_competitors)."""
    import ctypes as C

    import torch

    from oracle import oracle as O

    res = {}
    R = O.ref()
    s = torch.cuda.current_stream(dev)
    if R is not None:
        t, ln = C.c_int(), C.c_int()
        R.ref_tile_dims(A.nrow, A.nnz, 20, C.byref(t), C.byref(ln))
        tx = torch.zeros(t.value + 1, dtype=torch.int32, device=dev)
        ty = torch.zeros(t.value + 1, dtype=torch.int32, device=dev)
        desc = torch.zeros(max(ln.value, 1), dtype=torch.int64, device=dev)
        if R.ref_tile_build(20, rp.data_ptr(), A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(),
                            desc.data_ptr()) == 0:
            args = (0, col.data_ptr(), v.data_ptr(), A.nrow, A.nnz, tx.data_ptr(), ty.data_ptr(),
                    desc.data_ptr(), xd.data_ptr(), yd.data_ptr(), zd.data_ptr())
            R.ref_merbit_time_sigma(20, *args, 10, s.cuda_stream)
            ms = R.ref_merbit_time_sigma(20, *args, 200, s.cuda_stream)
            res["merbit_kernel_sigma20"] = {"value": round(B / (ms * 1e-3) / 1e9, 2),
                                            "unit": "GB/s", "ms_per_spmv": round(float(ms), 5)}
        del tx, ty, desc
    try:
        Acsr = torch.sparse_csr_tensor(rp, col, v, size=(A.nrow, A.ncol))
        for _ in range(3):
            torch.mv(Acsr, xd)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(50):
            torch.mv(Acsr, xd)
        e1.record(s)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 50
        res["cusparse_csr_spmv"] = {"value": round(B / (ms * 1e-3) / 1e9, 2), "unit": "GB/s",
                                    "ms_per_spmv": round(ms, 5),
                                    "via": "torch.mv on a torch.sparse_csr_tensor (cuSPARSE SpMV)"}
    except RuntimeError as e:  # a torch build without sparse CSR on CUDA
        res["cusparse_csr_spmv"] = {"unavailable": str(e).splitlines()[0][:120]}
    # the same in FP32 (values and x f32, 32-bit indices, cuSPARSE's plain
    # FP32 accumulation), beside this library's FP32 precision form
    try:
        A32 = torch.sparse_csr_tensor(rp, col, v.float(), size=(A.nrow, A.ncol))
        x32 = xd.float()
        for _ in range(3):
            torch.mv(A32, x32)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(50):
            torch.mv(A32, x32)
        e1.record(s)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / 50
        B32 = alg_bytes(A, "f32")
        res["cusparse_csr_spmv_f32"] = {"value": round(B32 / (ms * 1e-3) / 1e9, 2), "unit": "GB/s",
                                        "ms_per_spmv": round(ms, 5),
                                        "via": "torch.mv, FP32 values and x, int32 indices"}
        del A32, x32
    except RuntimeError as e:
        res["cusparse_csr_spmv_f32"] = {"unavailable": str(e).splitlines()[0][:120]}
    res.update(library_competitors(A, rp, col, v, xd, B, dev, y_cpu))
    return res


def library_competitors(A, rp, col, v, xd, B, dev, y_cpu, reps=50):
    """cuSPARSE CSR_ALG2 and COO_ALG2, CUB DeviceSpmv, CSR5 and HOLA, each
    called as the reference's src/spmv.cu calls it (oracle/competitors.cu).
    Each entry carries its normwise difference from the CPU FP64 product,
    max|y - y_cpu| / max|y_cpu|, to show that it computed the same SpMV."""
    import ctypes as C

    import torch

    from oracle import oracle as O

    L = O.comp()
    if L is None:
        return {}
    res = {}
    yc = torch.zeros(A.nrow, dtype=torch.float64, device=dev)
    scale = max(float(np.abs(y_cpu).max()), 1e-300) if A.nrow else 1.0
    ms, bms = C.c_float(), C.c_float()
    sigma = C.c_int()

    def record(name, rc, extra=None):
        if rc != 0:
            res[name] = {"error_code": int(rc)}
            return
        diff = float(np.abs(yc.cpu().numpy() - y_cpu).max()) / scale if A.nrow else 0.0
        res[name] = {"value": round(B / (ms.value * 1e-3) / 1e9, 2), "unit": "GB/s",
                     "ms_per_spmv": round(float(ms.value), 5),
                     "normwise_diff_vs_cpu_fp64": float(f"{diff:.3g}")}
        if extra:
            res[name].update(extra)
        yc.zero_()

    torch.cuda.synchronize(dev)
    rc = L.comp_cusparse_time(0, A.nrow, A.ncol, A.nnz, rp.data_ptr(), None, col.data_ptr(),
                              v.data_ptr(), xd.data_ptr(), yc.data_ptr(), reps, C.byref(ms))
    record("cusparse_csr_alg2", rc)
    counts = (rp[1:] - rp[:-1]).to(torch.int64)
    rows = torch.repeat_interleave(torch.arange(A.nrow, dtype=torch.int32, device=dev), counts,
                                   output_size=A.nnz)
    rc = L.comp_cusparse_time(1, A.nrow, A.ncol, A.nnz, rp.data_ptr(), rows.data_ptr(),
                              col.data_ptr(), v.data_ptr(), xd.data_ptr(), yc.data_ptr(), reps,
                              C.byref(ms))
    record("cusparse_coo_alg2", rc)
    del rows, counts
    rc = L.comp_cub_time(A.nrow, A.ncol, A.nnz, rp.data_ptr(), col.data_ptr(), v.data_ptr(),
                         xd.data_ptr(), yc.data_ptr(), reps, C.byref(ms))
    record("cub_device_spmv", rc)
    col_w, v_w = col.clone(), v.clone()  # CSR5 transposes these in place
    rc = L.comp_csr5_time(A.nrow, A.ncol, A.nnz, rp.data_ptr(), col_w.data_ptr(), v_w.data_ptr(),
                          xd.data_ptr(), yc.data_ptr(), reps, C.byref(bms), C.byref(ms),
                          C.byref(sigma))
    record("csr5", rc, {"sigma": sigma.value, "build_ms": round(float(bms.value), 3),
                        "timed": "memset of y + spmv per call, as the reference's loop"})
    del col_w, v_w
    rc = L.comp_hola_time(A.nrow, A.ncol, A.nnz, rp.data_ptr(), col.data_ptr(), v.data_ptr(),
                          xd.data_ptr(), yc.data_ptr(), reps, C.byref(bms), C.byref(ms))
    record("hola", rc, {"build_ms": round(float(bms.value), 3)})
    torch.cuda.synchronize(dev)
    return res


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload.startswith("rmat_batch"):
        run_batch(args)
    elif args.workload.endswith("_diff"):
        run_diff(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
