"""Benchmark: FP64 CSR SpMV HBM throughput on the large irregular matrix.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sbb|reference]
                    [--kernel merge|vector|tiled|auto] [--workload c2|c3|c1|c5]

Workload (default): the 5.5M-row irregular matrix (c2_circuit_5.5M: m = n =
5.5M, nnz ~ 60M, diagonal + band + power-law long-range entries, 550 dense
rows up to 1,000,000 nnz; val, x, y ~ U(-1,1); alpha = 1, beta = 0.5),
synthetic and seeded (the reference's SuiteSparse inputs are not available).

One step = one y = alpha*A*x + beta*y over the whole matrix with the data
resident in HBM.  ``value`` is algorithmic bytes / device time in GB/s,
bytes = 12*nnz + 4*(m+1) + 8*n + 16*m.  The working set (~874 MB) is larger
than L2 (126 MB), so no flush is done between steps.  ``e2e`` is the same
metric through the reference-facing C ABI (spMV_mgpu_v1, kernel 2) with host
buffers in pinned memory: every step copies the matrix, x and y to the GPU and
y back.  Multi-GPU runs are independent replicas (one per rank, no
collective); ``value`` sums the ranks' bytes over the slowest rank's time.
``library_spmv`` (one GPU) times cuSPARSE's SpMV, CSR ALG1 and ALG2, on the
same resident matrix after the timed region: the vendor library on the same
GPU, for context (``--no-library`` skips it).

``--workload c5`` prints the batched form's line instead: 512 seeded
matrices (banded / power-law / block-diagonal), each matrix's plain launches
one after another vs one CUDA graph over all of them (a persistent kernel per
kernel family on parallel branches, then one carry fix-up), with the
heuristic's and the exhaustive autotuner's kernel classes.

``--impl reference`` times the reference's host CSR SpMV (main.cu:350-356,
restated with +beta*y in oracle/sbb_oracle.c) on all host cores over a bounded
sample of the same workload; under torchrun only rank 0 runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sparse-blas_b200"))

import numpy as np  # noqa: E402

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}
KERNEL_TAGS = {1: "vector_kernel", 2: "merge_kernel", 3: "tiled_kernel", 5: "rows_kernel"}


def algo_bytes(m, n, nnz):
    return 12 * nnz + 4 * (m + 1) + 8 * n + 16 * m


def make_workload(name):
    from sbb import gen
    if name.startswith("mtx:"):  # a Matrix Market file (canonical CSR via the library's reader)
        from sbb import mmio
        A = mmio.read(name[4:])
        x = gen.uniform_vec(51, A.n)
        y = gen.uniform_vec(52, A.m)
        return A, x, y, 1.0, 0.5, (f"mtx {A.name}: {A.m} x {A.n}, nnz {A.nnz}, x and y U(-1,1) "
                                   "seeds 51/52, alpha=1, beta=0.5")
    if name == "c2":
        A = gen.c2()
        x = gen.uniform_vec(21, A.n)
        y = gen.uniform_vec(22, A.m)
        return A, x, y, 1.0, 0.5, "c2_circuit_5.5M: m=n=5,500,000, 550 dense rows (max 1,000,000 nnz), alpha=1, beta=0.5"
    if name == "c3":
        A = gen.c3()
        x = gen.uniform_vec(31, A.n)
        return A, x, np.zeros(A.m), 1.0, 0.0, "c3_shortwide: 4,284 x 1,092,610, lognormal rows (mean 2,640), val=1, alpha=1, beta=0"
    if name == "c1":
        A = gen.c1()
        x = gen.uniform_vec(11, A.n)
        return A, x, np.zeros(A.m), 1.0, 0.0, "c1_powerlaw_10k: n=10,000, power-law rows, alpha=1, beta=0"
    raise SystemExit(f"unknown workload {name}")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return PEAKS_FALLBACK["hbm_gbs"], "fallback"


def traffic_from_profile(kernel_tag, workload):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{kernel_tag}_{workload}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return int(float(line.split(":", 1)[1].strip()))
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        time.sleep(0.2)
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (getattr(self, "out", "") or "").splitlines():
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def max_over_ranks(v, ws):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_sample_time(A, x, y, alpha, beta, threads, budget_s=12.0):
    """Seconds per full pass of the reference's host loop (bounded sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    rp = np.ascontiguousarray(A.rowptr)
    reps, t_total = 0, 0.0
    # first pass also warms the page cache
    O.spmv_host(rp, A.col, A.val, x, alpha, beta, y, threads)
    while t_total < budget_s and reps < 50:
        t0 = time.perf_counter()
        O.spmv_host(rp, A.col, A.val, x, alpha, beta, y, threads)
        t_total += time.perf_counter() - t0
        reps += 1
    return t_total / reps, reps


def single_thread(A, x, y, alpha, beta, args):
    """The same host loop on one thread, as the reference runs it (a few
    seconds of passes)."""
    sec, reps = cpu_sample_time(A, x, y, alpha, beta, 1, budget_s=min(args.cpu_budget, 4.0))
    return {"value": round(algo_bytes(A.m, A.n, A.nnz) / sec / 1e9, 3), "unit": "GB/s",
            "cores": 1, "sample": f"{reps} full passes"}


def run_reference(args, ws, rank):
    """The reference's host CSR loop on all host cores: W warm-up passes and
    K timed passes over the same matrix as the GPU arm (each step one full
    SpMV), the timed passes stopped early only past two minutes."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    A, x, y, alpha, beta, desc = make_workload(args.workload)
    threads = os.cpu_count() or 1
    rp = np.ascontiguousarray(A.rowptr)
    for _ in range(max(args.warmup, 1)):
        O.spmv_host(rp, A.col, A.val, x, alpha, beta, y, threads)
    steps, t_total = 0, 0.0
    while steps < max(args.steps, 1) and t_total < 120.0:
        t0 = time.perf_counter()
        O.spmv_host(rp, A.col, A.val, x, alpha, beta, y, threads)
        t_total += time.perf_counter() - t0
        steps += 1
    sec = t_total / steps
    gbs = algo_bytes(A.m, A.n, A.nnz) / sec / 1e9
    one = single_thread(A, x, y, alpha, beta, args)
    line = {
        "metric": "SpMV HBM GB/s (FP64 CSR, algorithmic bytes 12*nnz+4*(m+1)+8*n+16*m)",
        "value": round(gbs, 3), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": steps, "warmup": max(args.warmup, 1), "ms_per_step": round(sec * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "GFLOP/s": round((2 * A.nnz + 3 * A.m) / sec / 1e9, 2),
        "config": {"workload": desc, "m": A.m, "n": A.n, "nnz": A.nnz,
                   "kernel": "host CSR loop (main.cu:350-356)", "threads": threads,
                   "parallelism": f"replicas x{args.gpus}"},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full passes of the host CSR loop (main.cu:350-356 "
                                   f"restated with +beta*y, OpenMP static over rows)",
                         "single_thread": one},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def default_class(A):
    """The plain path's heuristic on the batch classes (sbb.selector)."""
    from sbb.selector import heuristic_class
    return heuristic_class(A.rowptr)


BATCH_METRIC = ("batched SpMV GB/s (FP64 CSR matrices; one CUDA graph: a persistent kernel per "
                "kernel family + one carry fix-up)")
C5_DESC = ("c5: {count} matrices, n log-uniform [1k,200k], banded / power-law / block-diagonal "
           "thirds, nnz/row log-uniform [4,200], alpha=1, beta=0.5")


def c5_matrices(count, dev):
    """The batch: matrix i from seed 5+i, x and y from seeds 5000+i / 6000+i."""
    import torch
    from sbb import gen
    mats, total = [], 0
    for i in range(count):
        A = gen.c5(i)
        x = gen.uniform_vec(5000 + i, A.n)
        y = gen.uniform_vec(6000 + i, A.m)
        d = dict(m=A.m, n=A.n, alpha=1.0, beta=0.5, A=A, x_h=x, y_h=y)
        if dev is not None:
            d.update(rowptr=torch.from_numpy(A.rowptr32()).to(dev),
                     col=torch.from_numpy(A.col).to(dev), val=torch.from_numpy(A.val).to(dev),
                     x=torch.from_numpy(x).to(dev), y=torch.from_numpy(y).to(dev))
        total += algo_bytes(A.m, A.n, A.nnz)
        mats.append(d)
    return mats, total


def batch_measure(count, reps, local):
    """c5: `count` matrices; per-matrix plain launches vs one graph launch of
    the batch (a persistent kernel per kernel family, then the carry fix-up),
    with the learned selector's, the heuristic's and the exhaustive
    autotuner's classes.  Returns the measured figures (ms per batch, regrets,
    class counts); the batch with the selector's classes is the headline."""
    import torch
    from sbb.batch import Batch, tune
    from sbb.selector import Selector
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t_gen = time.perf_counter()
    mats, total_bytes = c5_matrices(count, dev)
    t_gen = time.perf_counter() - t_gen
    # exhaustive autotune: every class on every matrix, as plain launches
    t_tune = time.perf_counter()
    times = np.array([tune(d, reps=3) for d in mats])
    t_tune = time.perf_counter() - t_tune
    best = [int(np.argmin(t)) for t in times]
    default = [default_class(d["A"]) for d in mats]
    sel = Selector()
    t_sel = time.perf_counter()
    mlp = [sel.select(d) for d in mats]  # features, MLP and argmin on the GPU
    t_sel = time.perf_counter() - t_sel
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    res = {}
    for name, classes in (("mlp", mlp), ("default", default), ("tuned", best)):
        B = Batch(mats, classes)
        res[f"each_{name}_ms"] = timed(B.run_each, reps)
        res[f"batch_{name}_ms"] = timed(B.run_graph, reps)
        B.check()
        res[f"launches_each_{name}"] = B.launches(per_matrix=True)
        res[f"launches_batch_{name}"] = B.launches()
        B.close()
    best_sum = float(times.min(axis=1).sum())
    pick = lambda cls: float(sum(times[i, c] for i, c in enumerate(cls)))  # noqa: E731
    flops = sum(2 * d["A"].nnz + 3 * d["m"] for d in mats)
    del mats
    torch.cuda.empty_cache()
    return dict(res=res, total_bytes=total_bytes, flops=flops, t_gen=t_gen, t_tune=t_tune,
                t_sel=t_sel, mlp=mlp, best=best, default=default,
                regret_mlp=pick(mlp) / best_sum - 1, regret_default=pick(default) / best_sum - 1)


def run_batch(args, ws, rank, local):
    """c5 line: ``value`` is the batch with the selector's classes."""
    count = args.batch_count
    r = batch_measure(count, args.batch_reps, local)
    res, total_bytes = r["res"], r["total_bytes"]
    t_gen, t_tune, t_sel = r["t_gen"], r["t_tune"], r["t_sel"]
    mlp, best, default = r["mlp"], r["best"], r["default"]
    ms = max_over_ranks(res["batch_mlp_ms"], ws)
    value = total_bytes * ws / (ms * 1e-3) / 1e9
    if rank != 0:
        return
    line = {
        "metric": BATCH_METRIC,
        "value": round(value, 3), "unit": "GB/s", "n_gpus": ws, "steps": args.batch_reps,
        "warmup": 3, "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": C5_DESC.format(count=count),
                   "bytes_per_step": total_bytes, "l2_flush": "no (12.5 GB working set > L2)",
                   "classes": "selector (MLP) choices; per-matrix launches of the "
                              "heuristic's classes are the plain baseline",
                   "gen_s": round(t_gen, 1), "tune_s": round(t_tune, 1),
                   "select_s": round(t_sel, 2),
                   "classes_mlp": np.bincount(mlp, minlength=6).tolist(),
                   "classes_tuned": np.bincount(best, minlength=6).tolist(),
                   "classes_default": np.bincount(default, minlength=6).tolist(),
                   "speedup_batch_vs_each_default": round(res["each_default_ms"] / ms, 3),
                   "speedup_batch_vs_each_mlp": round(res["each_mlp_ms"] / ms, 3),
                   "regret_mlp": round(r["regret_mlp"], 4),
                   "regret_default": round(r["regret_default"], 4),
                   **{k: (round(v, 4) if isinstance(v, float) else v) for k, v in res.items()}},
        "gpu_launches": res["launches_batch_mlp"] * args.batch_reps,
    }
    print(json.dumps(line), flush=True)


def run_reference_batch(args, ws, rank):
    """The reference's host loop over the c5 matrices, all host cores, until
    the CPU budget is spent (bounded sample: the first k matrices)."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    mats, _ = c5_matrices(args.batch_count, None)
    done_bytes, t_total, k = 0, 0.0, 0
    for d in mats:
        A = d["A"]
        y = d["y_h"].copy()
        rp = np.ascontiguousarray(A.rowptr)
        t0 = time.perf_counter()
        O.spmv_host(rp, A.col, A.val, d["x_h"], 1.0, 0.5, y, threads)
        t_total += time.perf_counter() - t0
        done_bytes += algo_bytes(A.m, A.n, A.nnz)
        k += 1
        if t_total >= args.cpu_budget:
            break
    gbs = done_bytes / t_total / 1e9
    line = {
        "metric": BATCH_METRIC,
        "value": round(gbs, 3), "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": 1, "warmup": 0, "ms_per_step": round(t_total * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": C5_DESC.format(count=args.batch_count),
                                        "threads": threads},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"the first {k} matrices, one pass each"},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def f32_measure(A, x_h, y_h, alpha, beta, kernel, kw, warmup, steps, local, kernel64=None,
                kw64=None, lanes=True):
    """FP32-storage compensated form vs the FP64 plan on the same matrix, both
    timed here (main kernel with CUDA events, whole steps), with max and
    median per-row error against the FP64 double-double oracle.  kernel / kw
    configure the FP32 plan, kernel64 / kw64 the FP64 one (default: the
    same).  lanes: also the FP32-storage form with FP32 lane sums
    (sbb_plan_create_f32_lanes, 32 x 8 tiles), keys ``*_lanes``."""
    kernel64 = kernel if kernel64 is None else kernel64
    kw64 = kw if kw64 is None else kw64
    import ctypes as C
    import torch
    from sbb._lib import lib
    from sbb.device import Plan
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n = A.n
    rp = torch.from_numpy(A.rowptr32()).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    y0 = torch.from_numpy(y_h).to(dev)
    P64 = Plan(rp, col, torch.from_numpy(A.val).to(dev), n, kernel=kernel64, **kw64)
    P32 = Plan(rp, col, torch.from_numpy(A.val.astype(np.float32)).to(dev), n, kernel=kernel,
               f32=True, **kw)
    x64 = torch.from_numpy(x_h).to(dev)
    x32 = torch.from_numpy(x_h.astype(np.float32)).to(dev)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)

    def timed(P, x):
        y = y0.clone()
        for _ in range(warmup):
            P.spmv(x, y, alpha, beta)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * steps + 2)]
        for e in ev:
            e.record(stream)
        torch.cuda.synchronize()
        ev[0].record(stream)
        for i in range(steps):
            assert lib().sbb_spmv_timed(P.h, alpha, C.c_void_p(x.data_ptr()), beta,
                                        C.c_void_p(y.data_ptr()), sp,
                                        C.c_void_p(ev[2 + 2 * i].cuda_event),
                                        C.c_void_p(ev[3 + 2 * i].cuda_event)) == 0
        ev[1].record(stream)
        torch.cuda.synchronize()
        P.check()
        kern = statistics.median(ev[2 + 2 * i].elapsed_time(ev[3 + 2 * i]) for i in range(steps))
        return ev[0].elapsed_time(ev[1]) / steps, kern

    step64, kern64 = timed(P64, x64)
    step32, kern32 = timed(P32, x32)
    ref, sc = O.spmv_dd(A.rowptr, A.col, A.val, x_h, alpha, beta, y_h)

    def errors(P):
        y = y0.clone()
        P.spmv(x32, y, alpha, beta)
        torch.cuda.synchronize()
        err = np.abs(y.cpu().numpy() - ref) / np.where(sc > 0, sc, 1.0)
        return float(err.max()), float(np.median(err))

    err_max, err_median = errors(P32)
    info = P32.info()
    info64 = P64.info()
    launches = lib().sbb_plan_launches(P32.h)
    out = dict(step64=step64, kern64=kern64, step32=step32, kern32=kern32,
               err_max=err_max, err_median=err_median, info=info,
               info64=info64, launches=launches,
               tag=KERNEL_TAGS[info["kernel"]], tag64=KERNEL_TAGS[info64["kernel"]])
    if lanes:
        PL = Plan(rp, col, P32._keep[2], n, kernel="auto", f32=True, f32_lanes=True)
        out["step_lanes"], out["kern_lanes"] = timed(PL, x32)
        out["err_max_lanes"], out["err_median_lanes"] = errors(PL)
        out["sigma_lanes"] = PL.info()["tile_sigma"]
        PL.close()
    P64.close()
    P32.close()
    return out


def run_f32(args, ws, rank, local):
    """FP32-storage form line (``--f32``)."""
    A, x_h, y_h, alpha, beta, desc = make_workload(args.workload)
    m, n, nnz = A.m, A.n, A.nnz
    bytes64 = algo_bytes(m, n, nnz)
    bytes32 = 8 * nnz + 4 * (m + 1) + 4 * n + 16 * m
    # The FP64 side is the plain path as the default line runs it (the tiled
    # kernel, sigma 4); the FP32 side uses its own automatic choice (32 x 8
    # tiles) unless --kernel / --sigma say otherwise.
    kw = dict(tile_sigma=args.sigma) if args.kernel == "tiled" and args.sigma_given else {}
    kernel32 = args.kernel if args.sigma_given or args.kernel != "tiled" else "auto"
    with ClockSampler(local) as clk:
        r = f32_measure(A, x_h, y_h, alpha, beta, kernel32, kw, args.warmup, args.steps, local,
                        kernel64="tiled", kw64=dict(tile_sigma=4))
    ms32 = max_over_ranks(r["step32"], ws)
    peak, peak_kind = peaks()
    if rank == 0:
        ach = bytes32 / (r["kern32"] * 1e-3) / 1e9
        print(json.dumps({
            "metric": "SpMV GB/s, FP32-storage compensated form (algorithmic bytes "
                      "8*nnz+4*(m+1)+4*n+16*m)",
            "value": round(ws * bytes32 / (ms32 * 1e-3) / 1e9, 3), "unit": "GB/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms32, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": desc + " (val and x rounded to FP32, y FP64)", "m": m, "n": n,
                       "nnz": nnz, "kernel": r["tag"], "plan": {k: r["info"][k] for k in
                                                                ("tile_sigma", "vector_width",
                                                                 "items_per_thread")},
                       "fp64_kernel": r["tag64"], "fp64_tile_sigma": r["info64"]["tile_sigma"],
                       "fp64_plan_ms_per_step": round(r["step64"], 5),
                       "fp64_kernel_ms": round(r["kern64"], 5),
                       "f32_kernel_ms": round(r["kern32"], 5),
                       "speedup_step_vs_fp64": round(r["step64"] / r["step32"], 3),
                       "speedup_kernel_vs_fp64": round(r["kern64"] / r["kern32"], 3),
                       "byte_ratio": round(bytes64 / bytes32, 3),
                       "err_max": r["err_max"], "err_median": r["err_median"],
                       "err_metric": "|y - y_oracle| / (|alpha| sum|a x| + |beta y|), FP64 "
                                     "double-double oracle on the FP64 inputs",
                       "lanes": lanes_keys(r, bytes32, A)},
            "roofline": {"bound": "hbm", "achieved": round(ach, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(ach / peak, 4), "traffic": None, "peak_source": peak_kind},
            "gpu_launches": r["launches"] * args.steps,
            "clocks": clk.summary()}), flush=True)


def library_spmv(args, m, n, rp, col, val, x, y0, alpha, beta, bytes_step):
    """cuSPARSE's SpMV (CSR ALG1 and ALG2, the successors of the csrmv and
    csrmv_mp calls the reference makes) on the same resident matrix, timed
    with CUDA events on the same stream after the timed region: the vendor
    library's number on this GPU, for context; none of it is this library's
    work or counted in `value`."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    try:
        import cusparse_ref as CS
        stream = torch.cuda.current_stream()
        reps = max(3, min(args.steps, 200))
        out = {"impl": "cusparseSpMV, FP64 values, int32 indices, inputs resident"}
        for alg in ("alg1", "alg2"):
            y = y0.clone()
            op = CS.SpMV(m, n, rp, col, val, x, y, alg, stream)
            for _ in range(max(args.warmup, 3)):
                op.run(alpha, beta)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(reps):
                op.run(alpha, beta)
            e1.record(stream)
            torch.cuda.synchronize()
            op.close()
            ms = e0.elapsed_time(e1) / reps
            out[alg] = {"ms_per_call": round(ms, 5),
                        "GB/s": round(bytes_step / (ms * 1e-3) / 1e9, 2), "calls": reps}
        return out
    except Exception as e:  # a comparator only: its absence does not fail the bench
        return {"unavailable": f"{type(e).__name__}: {e}"}


def plain_measure(A, x_h, y_h, alpha, beta, kernel, kw, warmup, reps, local):
    """One plain plan on a resident matrix: the plan's build time (a second
    build, after the modules are loaded), the main kernel's median time and
    whole steps (kernel + carry fix-up), each over `reps` launches."""
    import ctypes as C
    import torch
    from sbb._lib import lib
    from sbb.device import Plan
    dev = torch.device("cuda", local)
    rp = torch.from_numpy(A.rowptr32()).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    val = torch.from_numpy(A.val).to(dev)
    x = torch.from_numpy(x_h).to(dev)
    y = torch.from_numpy(y_h).to(dev)
    Plan(rp, col, val, A.n, kernel=kernel, **kw).close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    P = Plan(rp, col, val, A.n, kernel=kernel, **kw)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    for _ in range(warmup):
        P.spmv(x, y, alpha, beta)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps + 2)]
    for e in ev:
        e.record(stream)
    torch.cuda.synchronize()
    ev[0].record(stream)
    for i in range(reps):
        assert lib().sbb_spmv_timed(P.h, alpha, C.c_void_p(x.data_ptr()), beta,
                                    C.c_void_p(y.data_ptr()), sp,
                                    C.c_void_p(ev[2 + 2 * i].cuda_event),
                                    C.c_void_p(ev[3 + 2 * i].cuda_event)) == 0
    ev[1].record(stream)
    torch.cuda.synchronize()
    P.check()
    kern = statistics.median(ev[2 + 2 * i].elapsed_time(ev[3 + 2 * i]) for i in range(reps))
    step = ev[0].elapsed_time(ev[1]) / reps
    graph = graph_step_ms(P, x, y, alpha, beta, min(reps, 100))
    info = P.info()
    launches = lib().sbb_plan_launches(P.h)
    P.close()
    return dict(kernel_ms=kern, step_ms=step, graph_step_ms=graph, plan_build_ms=build_ms,
                info=info, launches=launches)


def graph_step_ms(P, x, y, alpha, beta, steps):
    """ms per SpMV with `steps` SpMVs of the plan captured in one CUDA graph
    and replayed: the device time of a step without the host's launch work
    between steps (which dominates the host-launched step time of small
    matrices)."""
    import torch
    try:
        g = torch.cuda.CUDAGraph()
        cs = torch.cuda.Stream()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=cs):
            for _ in range(steps):
                P.spmv(x, y, alpha, beta)
        g.replay()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        del g
        return ms
    except Exception:  # a measurement aid only
        return None


def config_line(name, kernel, kw, local, cpu_budget, reps=200):
    """Sub-object of the default line for another benchmark configuration:
    GB/s and GFLOP/s of the step and of the main kernel, the fraction of the
    HBM peak, and the reference's host loop on the same matrix."""
    A, x_h, y_h, alpha, beta, desc = make_workload(name)
    r = plain_measure(A, x_h, y_h, alpha, beta, kernel, kw, 10, reps, local)
    b = algo_bytes(A.m, A.n, A.nnz)
    fl = 2 * A.nnz + 3 * A.m
    peak, peak_kind = peaks()
    threads = os.cpu_count() or 1
    sec, cpu_reps = cpu_sample_time(A, x_h, y_h, alpha, beta, threads, budget_s=cpu_budget)
    tag = KERNEL_TAGS[r["info"]["kernel"]]
    return {"workload": desc, "m": A.m, "n": A.n, "nnz": A.nnz, "kernel": tag,
            "plan": {k: r["info"][k] for k in ("vector_width", "items_per_thread",
                                               "tile_sigma", "tiles")},
            "step_ms": round(r["step_ms"], 5), "kernel_ms": round(r["kernel_ms"], 5),
            "graph_step_ms": (round(r["graph_step_ms"], 5) if r["graph_step_ms"] else None),
            "graph_GB/s": (round(b / (r["graph_step_ms"] * 1e-3) / 1e9, 2)
                           if r["graph_step_ms"] else None),
            "GB/s": round(b / (r["step_ms"] * 1e-3) / 1e9, 2),
            "GFLOP/s": round(fl / (r["step_ms"] * 1e-3) / 1e9, 2),
            "traffic": traffic_from_profile(tag, name),
            "kernel_GB/s": round(b / (r["kernel_ms"] * 1e-3) / 1e9, 2),
            "frac": round(b / (r["kernel_ms"] * 1e-3) / 1e9 / peak, 4), "peak": peak,
            "peak_source": peak_kind, "algorithmic_bytes": b, "flops": fl,
            "plan_build_ms": round(r["plan_build_ms"], 3), "reps": reps,
            "gpu_launches": r["launches"] * reps,
            "cpu_host_loop": {"GB/s": round(b / sec / 1e9, 3), "cores": threads,
                              "sample": f"{cpu_reps} full passes"}}


def lanes_keys(r, b32, A):
    """The FP32-lane-sum form's figures from f32_measure."""
    return {"api": "sbb_plan_create_f32_lanes", "tile_sigma": r["sigma_lanes"],
            "kernel_ms": round(r["kern_lanes"], 5), "step_ms": round(r["step_lanes"], 5),
            "speedup_kernel_vs_fp64": round(r["kern64"] / r["kern_lanes"], 3),
            "speedup_step_vs_fp64": round(r["step64"] / r["step_lanes"], 3),
            "GB/s": round(b32 / (r["step_lanes"] * 1e-3) / 1e9, 2),
            "kernel_GB/s": round(b32 / (r["kern_lanes"] * 1e-3) / 1e9, 2),
            "GFLOP/s": round((2 * A.nnz + 3 * A.m) / (r["step_lanes"] * 1e-3) / 1e9, 2),
            "err_max": r["err_max_lanes"], "err_median": r["err_median_lanes"]}


def extra_configs(A2, x2, y2, local, cpu_budget):
    """The other benchmark configurations, measured after the timed region of
    the default line (one GPU): c1 and c3 plain, the FP32-storage form on the
    c1 and c2 matrices (c4), and the 512-matrix batch with the learned
    selector (c5)."""
    out = {}
    out["c1"] = config_line("c1", "auto", {}, local, min(cpu_budget, 2.0), reps=500)
    out["c3"] = config_line("c3", "auto", {}, local, min(cpu_budget, 3.0), reps=100)
    f = {}
    for name, (A, x_h, y_h, alpha, beta) in (("c1_matrix", make_workload("c1")[:5]),
                                             ("c2_matrix", (A2, x2, y2, 1.0, 0.5))):
        r = f32_measure(A, x_h, y_h, alpha, beta, "auto", {}, 10, 100, local,
                        kernel64="tiled" if name == "c2_matrix" else "auto",
                        kw64=dict(tile_sigma=4) if name == "c2_matrix" else {})
        b64 = algo_bytes(A.m, A.n, A.nnz)
        b32 = 8 * A.nnz + 4 * (A.m + 1) + 4 * A.n + 16 * A.m
        f[name] = {"kernel": r["tag"], "tile_sigma": r["info"]["tile_sigma"],
                   "fp64_kernel": r["tag64"], "fp64_tile_sigma": r["info64"]["tile_sigma"],
                   "fp64_kernel_ms": round(r["kern64"], 5),
                   "f32_kernel_ms": round(r["kern32"], 5),
                   "fp64_step_ms": round(r["step64"], 5), "f32_step_ms": round(r["step32"], 5),
                   "speedup_kernel_vs_fp64": round(r["kern64"] / r["kern32"], 3),
                   "speedup_step_vs_fp64": round(r["step64"] / r["step32"], 3),
                   "f32_GB/s": round(b32 / (r["step32"] * 1e-3) / 1e9, 2),
                   "f32_GFLOP/s": round((2 * A.nnz + 3 * A.m) / (r["step32"] * 1e-3) / 1e9, 2),
                   "byte_ratio": round(b64 / b32, 3),
                   "err_max": r["err_max"], "err_median": r["err_median"],
                   "lanes": lanes_keys(r, b32, A)}
    f["err_metric"] = ("|y - y_oracle| / (|alpha| sum|a x| + |beta y|) against the FP64 "
                       "double-double oracle on the FP64 inputs")
    out["f32"] = f
    r = batch_measure(512, 10, local)
    res = r["res"]
    ms = res["batch_mlp_ms"]
    out["c5"] = {"workload": C5_DESC.format(count=512),
                 "batch_ms": round(ms, 4), "each_ms": round(res["each_default_ms"], 4),
                 "speedup_batch_vs_each": round(res["each_default_ms"] / ms, 3),
                 "batch_tuned_ms": round(res["batch_tuned_ms"], 4),
                 "batch_default_ms": round(res["batch_default_ms"], 4),
                 "GB/s": round(r["total_bytes"] / (ms * 1e-3) / 1e9, 2),
                 "GFLOP/s": round(r["flops"] / (ms * 1e-3) / 1e9, 2),
                 "regret_mlp": round(r["regret_mlp"], 4),
                 "regret_default": round(r["regret_default"], 4),
                 "launches_batch": res["launches_batch_mlp"],
                 "launches_each": res["launches_each_default"],
                 "baseline": "each matrix's own plain launches with the heuristic's classes"}
    return out


def run_sbb(args, ws, rank, local):
    import ctypes as C
    import torch
    from sbb._lib import lib
    from sbb.device import Plan
    from sbb import api

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    A, x_h, y_h, alpha, beta, desc = make_workload(args.workload)
    m, n, nnz = A.m, A.n, A.nnz
    bytes_step = algo_bytes(m, n, nnz)

    rp = torch.from_numpy(A.rowptr32()).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    val = torch.from_numpy(A.val).to(dev)
    x = torch.from_numpy(x_h).to(dev)
    y0 = torch.from_numpy(y_h).to(dev)
    y = y0.clone()
    kw = {}
    if args.kernel == "merge":
        kw = dict(items_per_thread=args.ipt, persistent=args.persistent)
    elif args.kernel == "tiled":
        kw = dict(tile_sigma=args.sigma)
    P = Plan(rp, col, val, n, kernel=args.kernel, **kw)
    info = P.info()
    launches = lib().sbb_plan_launches(P.h)
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)

    # warm-up
    for _ in range(args.warmup):
        P.spmv(x, y, alpha, beta)
    torch.cuda.synchronize()
    P.check()

    # timed region: whole steps (value) and the main kernel alone (roofline)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for e in starts + stops:  # torch creates the CUDA event on first record
        e.record(stream)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier(ws)
        torch.cuda.synchronize()
        t0.record(stream)
        for i in range(args.steps):
            rc = lib().sbb_spmv_timed(P.h, alpha, C.c_void_p(x.data_ptr()), beta,
                                      C.c_void_p(y.data_ptr()), sp,
                                      C.c_void_p(starts[i].cuda_event),
                                      C.c_void_p(stops[i].cuda_event))
            assert rc == 0
        t1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
    P.check()
    ms_total = t0.elapsed_time(t1)
    ms_step = max_over_ranks(ms_total / args.steps, ws)
    kern_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    kern_avg = statistics.mean(kern_ms)
    value = ws * bytes_step / (ms_step * 1e-3) / 1e9

    # The same steps as a caller runs them, with no events between the main
    # kernel and the carry fix-up (an event there keeps the fix-up, a
    # programmatic dependent launch, from starting before the kernel ends).
    u0 = torch.cuda.Event(enable_timing=True)
    u1 = torch.cuda.Event(enable_timing=True)
    barrier(ws)
    torch.cuda.synchronize()
    u0.record(stream)
    for _ in range(args.steps):
        P.spmv(x, y, alpha, beta)
    u1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    P.check()
    ms_plain = max_over_ranks(u0.elapsed_time(u1) / args.steps, ws)
    peak, peak_kind = peaks()
    achieved = bytes_step / (kern_avg * 1e-3) / 1e9
    tag = KERNEL_TAGS[info["kernel"]]
    traffic = traffic_from_profile(tag, args.workload) if not args.workload.startswith("mtx:") else None

    # e2e through the reference-facing C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        pinned = {}

        def pin(a):
            t_ = torch.from_numpy(a).pin_memory()
            arr = t_.numpy()
            pinned[id(arr)] = t_
            return arr
        rp64, colp, valp, xp = pin(A.rowptr), pin(A.col), pin(A.val), pin(x_h)
        yp = pin(y_h.copy())
        for _ in range(2):
            yp[:] = y_h
            assert api.spMV_mgpu_v1(m, n, nnz, alpha, valp, rp64, colp, xp, beta, yp, 1, 2) == 0
        e_steps = max(3, min(args.steps, 10))
        h2d = 8 * (m + 1) + 4 * nnz + 8 * nnz + 8 * n + (8 * m if beta != 0 else 0)
        # This box's PCIe floor: the same bytes as plain pinned copies (host
        # to device, then y back), timed after each call so that both see the
        # same moment of the host's and the link's other traffic.
        src = [pinned[id(a)] for a in (rp64, colp, valp, xp) + ((yp,) if beta != 0 else ())]
        dst = [torch.empty_like(t_, device=dev) for t_ in src]
        yback = pinned[id(yp)]
        ydev = torch.zeros_like(yback, device=dev)
        call_s, copy_s, phases = [], [], []
        ph = (C.c_double * 5)()
        barrier(ws)
        torch.cuda.synchronize()
        for _ in range(e_steps):
            tt = time.perf_counter()
            rc = api.spMV_mgpu_v1(m, n, nnz, alpha, valp, rp64, colp, xp, beta, yp, 1, 2)
            call_s.append(time.perf_counter() - tt)
            assert rc == 0
            if lib().sbb_last_call_phases(ph, 5) == 5:
                phases.append(list(ph))
            tt = time.perf_counter()
            for d_, s_ in zip(dst, src):
                d_.copy_(s_, non_blocking=True)
            yback.copy_(ydev, non_blocking=True)
            torch.cuda.synchronize()
            copy_s.append(time.perf_counter() - tt)
        # The same copies with y going back on a second stream while the
        # matrix goes in (both directions of the link at once, as the call's
        # chunked pipeline does).
        both_s = []
        side = torch.cuda.Stream()
        for _ in range(e_steps):
            torch.cuda.synchronize()
            tt = time.perf_counter()
            with torch.cuda.stream(side):
                yback.copy_(ydev, non_blocking=True)
            for d_, s_ in zip(dst, src):
                d_.copy_(s_, non_blocking=True)
            torch.cuda.synchronize()
            both_s.append(time.perf_counter() - tt)
        yp[:] = y_h  # the floor's copy back overwrote the host y
        e_sec = max_over_ranks(sum(call_s) / e_steps, ws)
        c_sec = max_over_ranks(sum(copy_s) / e_steps, ws)
        del dst, ydev
        spread = lambda v: {"min": round(min(v) * 1e3, 3),  # noqa: E731
                            "median": round(statistics.median(v) * 1e3, 3),
                            "max": round(max(v) * 1e3, 3)}
        e2e = {"value": round(ws * bytes_step / e_sec / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 8 * m,
               "ms_per_step": round(e_sec * 1e3, 3),
               "pcie_copy_floor_ms": round(c_sec * 1e3, 3),
               "call_ms": spread(call_s), "pcie_copy_floor_call_ms": spread(copy_s),
               "pcie_copy_both_directions_ms": spread(both_s),
               "call_phases_ms_median": (dict(zip(
                   ("host_prep", "rowptr_check_wait", "plans_and_launches", "kernels_and_copy_back",
                    "host_merges"),
                   [round(statistics.median(p_[i] for p_ in phases), 3) for i in range(5)]))
                   if phases else None),
               "api": "spMV_mgpu_v1(kernel=2) host pointers, pinned",
               "note": "the host-pointer call copies the whole matrix, x and y over PCIe in "
                       "every step (most of the step), so it runs the merge-path kernel "
                       "(kernel 2, a cheap plan per call); value and roofline are the tiled "
                       "kernel on resident data"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        sec, reps = cpu_sample_time(A, x_h, y_h, alpha, beta, threads, budget_s=args.cpu_budget)
        cpu = {"value": round(bytes_step / sec / 1e9, 3), "unit": "GB/s", "cores": threads,
               "kind": "port",
               "sample": f"{reps} full passes of the host CSR loop over this matrix "
                         f"(main.cu:350-356 restated with +beta*y; OpenMP static)",
               "single_thread": single_thread(A, x_h, y_h, alpha, beta, args)}

    library = None
    if rank == 0 and ws == 1 and not args.no_library:
        library = library_spmv(args, m, n, rp, col, val, x, y0, alpha, beta, bytes_step)

    # one-time costs: the plan build (a second build of the same plan) and the
    # reference-named csr5_kernel, which builds and drops a tile plan per call
    build = None
    if rank == 0 and ws == 1 and not args.no_extra:
        torch.cuda.synchronize()
        t_b = time.perf_counter()
        P2 = Plan(rp, col, val, n, kernel=args.kernel, **kw)
        torch.cuda.synchronize()
        build_ms = (time.perf_counter() - t_b) * 1e3
        P2.close()
        a_c, b_c = C.c_double(alpha), C.c_double(beta)
        yc = y0.clone()
        csr5 = []
        for _ in range(4):
            torch.cuda.synchronize()
            t_c = time.perf_counter()
            rc = lib().csr5_kernel(m, n, nnz, C.byref(a_c), C.c_void_p(val.data_ptr()),
                                   C.c_void_p(rp.data_ptr()), C.c_void_p(col.data_ptr()),
                                   C.c_void_p(x.data_ptr()), C.byref(b_c),
                                   C.c_void_p(yc.data_ptr()))
            torch.cuda.synchronize()
            csr5.append((time.perf_counter() - t_c) * 1e3)
            assert rc == 0
        build = {"plan_build_ms": round(build_ms, 3),
                 "break_even_spmv_vs_cusparse_alg1": (
                     round(build_ms / (library["alg1"]["ms_per_call"] - ms_step), 1)
                     if library and "alg1" in library
                     and library["alg1"]["ms_per_call"] > ms_step else None),
                 "csr5_kernel_ms_per_call": round(statistics.median(csr5[1:]), 3),
                 "note": "plan_build_ms: host wall time of a second sbb_plan_create of the "
                         "timed plan (row-pointer check, tile format, carry lists); "
                         "csr5_kernel (device pointers) builds, runs and drops a tile plan "
                         "in every call, as the reference converts to CSR5 in every call"}

    extra = {}
    if rank == 0 and ws == 1 and args.workload == "c2" and not args.no_extra:
        with ClockSampler(local) as clk2:
            extra = extra_configs(A, x_h, y_h, local, args.cpu_budget)
        extra["extra_clocks"] = clk2.summary()

    if rank == 0:
        line = {
            "metric": "SpMV HBM GB/s (FP64 CSR, algorithmic bytes 12*nnz+4*(m+1)+8*n+16*m)",
            "value": round(value, 3), "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "m": m, "n": n, "nnz": nnz,
                       "kernel": tag, "plan": {k: info[k] for k in
                                               ("items_per_thread", "persistent", "tile_sigma",
                                                "vector_width", "tiles")},
                       "l2": "inputs larger than L2 (working set %.0f MB), no flush" % (bytes_step / 1e6),
                       "parallelism": f"replicas x{ws}"},
            "GFLOP/s": round(ws * (2 * nnz + 3 * m) / (ms_step * 1e-3) / 1e9, 2),
            "kernel_GFLOP/s": round((2 * nnz + 3 * m) / (kern_avg * 1e-3) / 1e9, 2),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_source": peak_kind,
                         "kernel_ms_avg": round(kern_avg, 5),
                         "kernel_ms_median": round(statistics.median(kern_ms), 5),
                         "algorithmic_bytes_per_launch": bytes_step},
            "steps_without_kernel_events": {
                "ms_per_step": round(ms_plain, 5),
                "GB/s": round(ws * bytes_step / (ms_plain * 1e-3) / 1e9, 3),
                "note": "the timed steps above record CUDA events around the main kernel; "
                        "these steps (same count, after them) do not"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "library_spmv": library,
            "one_time": build,
            **extra,
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    P.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="sbb", choices=["sbb", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c5"])
    ap.add_argument("--mtx", default=None, help="benchmark a Matrix Market file instead")
    ap.add_argument("--batch-count", type=int, default=512, help="c5: matrices in the batch")
    ap.add_argument("--batch-reps", type=int, default=20, help="c5: timed batch runs")
    ap.add_argument("--kernel", default="tiled",
                    choices=["merge", "vector", "tiled", "rows", "auto"])
    ap.add_argument("--ipt", type=int, default=6)
    ap.add_argument("--persistent", type=int, default=0)
    ap.add_argument("--sigma", type=int, default=None,
                    help="tiled kernel: nnz per lane (0 = CSR5 rule; default 4)")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-library", action="store_true",
                    help="skip the cuSPARSE comparator (library_spmv key)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the one-time costs and (c2) the c1 / c3 / FP32 / c5 sub-objects")
    ap.add_argument("--f32", action="store_true",
                    help="time the FP32-storage compensated form against the FP64 plan")
    args = ap.parse_args()
    args.sigma_given = args.sigma is not None
    if args.sigma is None:
        args.sigma = 4
    if args.warmup < 3:
        args.warmup = 3
    if args.mtx:
        args.workload = "mtx:" + os.path.abspath(args.mtx)
    ws, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            (run_reference_batch if args.workload == "c5" else run_reference)(args, ws, rank)
        elif args.workload == "c5":
            run_batch(args, ws, rank, local)
        elif args.f32:
            run_f32(args, ws, rank, local)
        else:
            run_sbb(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
