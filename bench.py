#!/usr/bin/env python
"""Benchmark of the SpMV hot path on B200.

Headline: SpMV HBM GB/s, CSR FP64, 3-D 7-point Dirichlet Laplacian on a
128^3 grid (n = 2,097,152, nnz = 14,581,760), the SpMV format-sweep
configuration.  A step is one product y = A x.

  value     algorithmic bytes of one product / device time per step
            (CUDA events on the launching stream, inputs resident in HBM;
            the matrix, x and y are 217 MB, above the 126 MB L2)
  e2e       the same metric through the drop-in call sk_spmv_host, with x
            copied in from pinned host memory and y copied back every step
  roofline  dominant kernel vs the measured HBM copy bandwidth
  cpu_baseline  the reference's own multiply (oracle/_ref, compiled from
            its sources) on 1 host core over a bounded sample
  sweep     GB/s of every format / precision on the sweep matrices

--impl reference times the reference's CPU multiply with all host threads
(rank 0 only).  Under torchrun every rank runs an independent replica of
the workload (the path has no exchange step), and the slowest rank's time
is used.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

HBM_FALLBACK_GBS = 6650.0
L2_BYTES = 126 * 1024 * 1024
WORKLOAD = "SpMV CSR FP64, 3-D 7-point Dirichlet Laplacian 128^3 (n=2097152, nnz=14581760)"
METRIC = "SpMV HBM GB/s (CSR FP64, 7-point Laplacian 128^3)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20000)
    p.add_argument("--warmup", type=int, default=200)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--grid", type=int, default=128)
    p.add_argument("--no-sweep", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--profile-formats", action="store_true",
                   help="run one product of every sweep format and precision (for ncu captures), no timing")
    return p.parse_args()


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def profiled_traffic(tag):
    """Per-launch DRAM bytes of kernel `tag` from the committed ncu summary
    (a line `traffic[<tag>]: <bytes>` in profiles/*.md), else None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    key = f"traffic[{tag}]:"
    for name in sorted(os.listdir(pdir)):
        if not name.endswith((".md", ".txt")):
            continue
        with open(os.path.join(pdir, name)) as f:
            for line in f:
                if key in line:
                    try:
                        return int(float(line.split(key, 1)[1].split()[0]))
                    except ValueError:
                        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", device_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_workload(grid):
    from sparkit_b200 import matgen
    A = matgen.laplacian_3d_dirichlet(grid)
    x = matgen.uniform_vector(A.shape()[0], seed=1)
    return A, x


# ---------------------------------------------------------------------
# the reference arm
# ---------------------------------------------------------------------
def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    from oracle.binding import Oracle, Reference, reference_available
    from sparkit_b200 import formats
    A, x = build_workload(args.grid)
    n = A.shape()[0]
    nthreads = os.cpu_count() or 1
    # each step: every host thread runs the reference multiply on a row
    # slice of A sized so that the whole run stays within ~2 minutes
    total = args.steps + args.warmup
    budget_s = 90.0
    per_row_s = 16e-9  # about 16 ns per row on one core (measured order)
    rows = int(min(n, max(args.grid * args.grid, budget_s / max(total, 1) / per_row_s)))
    rp = A.row_ptr()[: rows + 1].copy()
    S = formats.Compressed_row_matrix((rows, n), rp, A.col_ind()[: rp[-1]], A.values()[: rp[-1]])
    if reference_available():
        R = Reference()
        kind = "reference"
        h_seconds = lambda k: R.multiply_threads_seconds(S, x, nthreads, k)  # noqa: E731
    else:
        O = Oracle()
        kind = "port"
        import concurrent.futures as cf
        pool = cf.ThreadPoolExecutor(nthreads)

        def h_seconds(k):
            t0 = time.perf_counter()
            list(pool.map(lambda _: [O.spmv(S, x) for _ in range(k)], range(nthreads)))
            return time.perf_counter() - t0
    for _ in range(max(args.warmup, 0)):
        h_seconds(1)
    secs = h_seconds(max(args.steps, 1))
    nnz = int(rp[-1])
    bytes_one = 8 * nnz + 4 * nnz + 4 * (rows + 1) + 8 * n + 8 * rows
    gbs = bytes_one * nthreads * max(args.steps, 1) / secs / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / max(args.steps, 1) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 7-point Laplacian, x ~ U[-1,1] seed 1)",
        "config": {"workload": WORKLOAD, "sample_rows": rows, "threads": nthreads},
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": nthreads, "kind": kind,
                         "sample": f"rows 0..{rows} of the 128^3 matrix, one reference multiply per thread per "
                                   f"step, {nthreads} threads concurrently; int32-index byte model"},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------
def time_device(fn, steps, warmup, stream):
    import torch
    torch.cuda.synchronize()
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps  # ms per step


def sweep(stream, grid):
    """GB/s of each format and precision (algorithmic bytes / event time)."""
    import torch

    from sparkit_b200 import formats, gpu, matgen
    out = {}
    sptr = gpu.torch_stream(stream)
    A, x = build_workload(grid)
    for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
        Adt = A.astype(dt)
        xd = torch.from_numpy(x.astype(dt)).cuda()
        yd = torch.empty_like(xd)
        for fmt, M in (("csr", Adt), ("ell", formats.to_ellpack(Adt)), ("jad", formats.to_jagged_diagonal(Adt))):
            Ad = gpu.Device_matrix(M)
            ms = time_device(lambda: Ad.spmv(xd, yd, stream=sptr), 300, 20, stream)
            out[f"lap3d_{fmt}_{tag}"] = {"gbs": Ad.info()["spmv_bytes"] / ms / 1e6, "us": ms * 1e3}
            Ad.close()
    del A
    B = matgen.vector_laplacian_3d_bsr(grid, seed=1)
    Bd = gpu.Device_matrix(B)
    xb = torch.from_numpy(matgen.uniform_vector(B.shape()[0], seed=2)).cuda()
    yb = torch.empty_like(xb)
    ms = time_device(lambda: Bd.spmv(xb, yb, stream=sptr), 200, 20, stream)
    out["vec3_bsr33_f64"] = {"gbs": Bd.info()["spmv_bytes"] / ms / 1e6, "us": ms * 1e3}
    Bd.close()
    del B
    Z = matgen.zipf_random(1_000_000, s=1.5, cap=2048, seed=0)
    Zd = gpu.Device_matrix(Z)
    xz = torch.from_numpy(matgen.uniform_vector(Z.shape()[0], seed=3)).cuda()
    yz = torch.empty_like(xz)
    ms = time_device(lambda: Zd.spmv(xz, yz, stream=sptr), 200, 20, stream)
    out["zipf_csr_f64"] = {"gbs": Zd.info()["spmv_bytes"] / ms / 1e6, "us": ms * 1e3, "nnz": Z.size(),
                           "mean_row": Z.size() / Z.shape()[0]}
    return out


def cpu_baseline(A, x, bytes_one):
    """The reference's own multiply (oracle/_ref) on one host core, over a
    bounded number of full products; falls back to the C oracle port."""
    from oracle.binding import Oracle, Reference, reference_available
    if reference_available():
        R = Reference()
        t1 = R.multiply_threads_seconds(A, x, 1, 1)
        reps = int(max(3, min(200, 10.0 / max(t1, 1e-3))))
        secs = R.multiply_threads_seconds(A, x, 1, reps)
        kind = "reference"
    else:
        O = Oracle()
        t0 = time.perf_counter()
        O.spmv(A, x)
        t1 = time.perf_counter() - t0
        reps = int(max(3, min(200, 10.0 / max(t1, 1e-3))))
        t0 = time.perf_counter()
        for _ in range(reps):
            O.spmv(A, x)
        secs = time.perf_counter() - t0
        kind = "port"
    return {"value": bytes_one * reps / secs / 1e9, "unit": "GB/s", "cores": 1, "kind": kind,
            "sample": f"{reps} full products of the 128^3 matrix on one core (~{secs:.1f} s), "
                      f"same int32-index byte model as the GPU figure", "ms_per_product": secs / reps * 1e3}


def profile_formats(grid):
    """One product per sweep format / precision, for an ncu capture that
    selects the kernels by name (-k regex:spmv)."""
    import torch

    from sparkit_b200 import formats, gpu, matgen
    torch.cuda.set_device(0)
    A, x = build_workload(grid)
    for dt in (np.float64, np.float32):
        Adt = A.astype(dt)
        xd = torch.from_numpy(x.astype(dt)).cuda()
        yd = torch.empty_like(xd)
        for M in (Adt, formats.to_ellpack(Adt), formats.to_jagged_diagonal(Adt)):
            Ad = gpu.Device_matrix(M)
            Ad.spmv(xd, yd)
            torch.cuda.synchronize()
            Ad.close()
    B = matgen.vector_laplacian_3d_bsr(grid // 2, seed=1)
    Bd = gpu.Device_matrix(B)
    xb = torch.from_numpy(matgen.uniform_vector(B.shape()[0], seed=2)).cuda()
    Bd.spmv(xb, torch.empty_like(xb))
    Z = matgen.zipf_random(250_000, s=1.5, cap=2048, seed=0)
    Zd = gpu.Device_matrix(Z)
    xz = torch.from_numpy(matgen.uniform_vector(Z.shape()[0], seed=3)).cuda()
    Zd.spmv(xz, torch.empty_like(xz))
    torch.cuda.synchronize()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_formats:
        return profile_formats(args.grid)
    import torch
    world, rank, local = dist_setup()
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    from sparkit_b200 import _lib, gpu
    dev = torch.cuda.current_device()
    # a dedicated stream: the kernels and the CUDA events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = gpu.torch_stream(stream)

    A, x = build_workload(args.grid)
    n = A.shape()[0]
    Ad = gpu.Device_matrix(A)
    info = Ad.info()
    bytes_one = info["spmv_bytes"]
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)

    def step():
        Ad.spmv(xd, yd, stream=sptr)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        dev_id = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
    except Exception:
        dev_id = str(dev)
    sampler = ClockSampler(dev_id)
    time.sleep(0.3)
    launches0 = _lib.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    launches = _lib.launch_count() - launches0
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = bytes_one * world / (ms * 1e-3) / 1e9

    # e2e through the drop-in host call, pinned host buffers
    xh = torch.from_numpy(x).pin_memory()
    yh = torch.empty(n, dtype=torch.float64).pin_memory()
    xp, yp = ctypes.c_void_p(xh.data_ptr()), ctypes.c_void_p(yh.data_ptr())
    L = _lib.lib()
    e2e_steps = max(20, min(args.steps // 20, 500))
    for _ in range(5):
        _lib.check(L.sk_spmv_host(Ad.handle, xp, yp))
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        _lib.check(L.sk_spmv_host(Ad.handle, xp, yp))
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    y_host = yh.numpy()
    assert np.isfinite(y_host).all()

    peak, peak_kind = measured_peak()
    achieved = bytes_one / (ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6650 GB/s",
                "traffic": profiled_traffic("csr_spmv_f64_lap3d128"),
                "kernel": "csr_spmv_kernel<double, EpiStore<double>>",
                "bytes_model": "8*nnz + 4*nnz + 4*(n+1) + 8*n (x) + 8*n (y)", "bytes_per_launch": bytes_one}

    extra = {}
    if rank == 0 and world == 1 and not args.no_cpu:
        extra["cpu_baseline"] = cpu_baseline(A, x, bytes_one)
    if rank == 0 and world == 1 and not args.no_sweep:
        Ad.close()
        extra["sweep"] = sweep(stream, args.grid)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 7-point Dirichlet Laplacian, x ~ U[-1,1] seed 1)",
            "config": {"workload": WORKLOAD, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": f"inputs {bytes_one / 1e6:.0f} MB per product > 126 MB L2, no flush"},
            "e2e": {"value": bytes_one * world / e2e_s / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "ms_per_step": e2e_s * 1e3, "call": "sk_spmv_host (pinned host x, y)"},
            "roofline": roofline,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
