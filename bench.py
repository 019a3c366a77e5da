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
    p.add_argument("--no-solvers", action="store_true")
    p.add_argument("--profile-solvers", action="store_true",
                   help="run 20 FP64 and 20 FP32 CG iterations on the GRF diffusion matrix (for ncu launch lists)")
    p.add_argument("--profile-learned", action="store_true",
                   help="apply the (untrained) learned preconditioner on 512^2 four times, for ncu")
    p.add_argument("--profile-gmres", action="store_true",
                   help="40 iterations of GMRES(30) on the 1024^2 convection-diffusion problem (for ncu)")
    p.add_argument("--profile-mixed-diagonals", action="store_true",
                   help="the --profile-mixed run on a handle with its diagonal copy")
    p.add_argument("--profile-mixed", action="store_true",
                   help="one mixed solve with 100 persistent FP32 inner iterations on the 128^3 GRF problem, for ncu")
    p.add_argument("--no-convert", action="store_true")
    p.add_argument("--no-eigen", action="store_true")
    p.add_argument("--no-mm", action="store_true")
    p.add_argument("--profile-eigen", action="store_true",
                   help="one sk_eigenvalue_bounds on the grid^3 Laplacian (for an ncu launch list)")
    p.add_argument("--profile-convert", action="store_true",
                   help="each device format conversion once (for an ncu launch list)")
    p.add_argument("--profile-zipf", action="store_true",
                   help="three CSR FP64 products of matrix B (1M rows, Zipf(1.5) lengths), for ncu")
    p.add_argument("--profile-zipf-panels", action="store_true",
                   help="the --profile-zipf products on the handle's column-panel copy")
    p.add_argument("--profile-formats", action="store_true",
                   help="run one product of every sweep format and precision (for ncu captures), no timing")
    p.add_argument("--profile-small-solves", action="store_true",
                   help="the one-launch FP64 solves twice each: Jacobi-CG on the 256^2 Laplacian, then Jacobi "
                        "BiCGSTAB, CGS and MINRES (for ncu)")
    p.add_argument("--profile-batched", action="store_true",
                   help="the batched CG on 512 of the 4096 systems, twice (for ncu)")
    p.add_argument("--profile-c4", action="store_true",
                   help="60 FGMRES(30) iterations with the two-level preconditioner and an untrained network "
                        "smoother on the 512^2 problem, then 60 with two-level Jacobi (for an ncu launch list)")
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
    h0 = time.perf_counter()
    for _ in range(warmup):
        fn()
    host_per_call = (time.perf_counter() - h0) / max(warmup, 1)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        torch.cuda._sleep(int(min(0.25, 1.5 * host_per_call * min(steps, 1000)) * 2.0e9))
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
        # the FP32 diagonal copy with x and y (80 MB at 128^3) would sit in
        # the L2 between products, so the copy is timed in FP64 only (155 MB)
        for fmt, M in (("csr", Adt), ("ell", formats.to_ellpack(Adt)), ("jad", formats.to_jagged_diagonal(Adt)),
                       ("csr_diagonal_copy", Adt if tag == "f64" else None)):
            if M is None:
                continue
            Ad = gpu.Device_matrix(M)
            if fmt == "csr_diagonal_copy":
                assert Ad.add_diagonals()
            ms = time_device(lambda: Ad.spmv(xd, yd, stream=sptr), 300, 20, stream)
            # spmv_bytes is the byte model of the layout the product reads
            # (for the diagonal copy: its values and row masks, x and y)
            info = Ad.info()
            out[f"lap3d_{fmt}_{tag}"] = {"gbs": info["spmv_bytes"] / ms / 1e6, "us": ms * 1e3,
                                         "bytes": info["spmv_bytes"], "layout": Ad.layout(),
                                         "device_bytes": info["device_bytes"]}
            Ad.close()
    del A
    B = matgen.vector_laplacian_3d_bsr(grid, seed=1)
    for tag, dt in (("f64", np.float64), ("f32", np.float32)):
        Bd = gpu.Device_matrix(B, dtype=dt)
        xb = torch.from_numpy(matgen.uniform_vector(B.shape()[0], seed=2, dtype=dt)).cuda()
        yb = torch.empty_like(xb)
        ms = time_device(lambda: Bd.spmv(xb, yb, stream=sptr), 200, 20, stream)
        out[f"vec3_bsr33_{tag}"] = {"gbs": Bd.info()["spmv_bytes"] / ms / 1e6, "us": ms * 1e3}
        Bd.close()
    del B
    # matrix B: CSR, and JAD and ELL built on the device from the CSR handle
    # (the ELL holds 2048 slots per row, 2.05e9 slots; its byte model counts
    # the stored entries only), FP64 and FP32
    Z = matgen.zipf_random(1_000_000, s=1.5, cap=2048, seed=0)
    for tag, dt in (("f64", np.float64), ("f32", np.float32)):
        t0 = time.perf_counter()
        Zd = gpu.Device_matrix(Z, dtype=dt)
        upload_s = time.perf_counter() - t0
        xz = torch.from_numpy(matgen.uniform_vector(Z.shape()[0], seed=3, dtype=dt)).cuda()
        yz = torch.empty_like(xz)
        ms = time_device(lambda: Zd.spmv(xz, yz, stream=sptr), 200, 20, stream)
        info = Zd.info()
        csr_bytes = (8 if dt == np.float64 else 4) * Z.size() + 4 * Z.size() + 4 * (Z.shape()[0] + 1)
        out[f"zipf_csr_{tag}"] = {"gbs": info["spmv_bytes"] / ms / 1e6, "us": ms * 1e3, "nnz": Z.size(),
                                  "mean_row": Z.size() / Z.shape()[0], "layout": Zd.layout(),
                                  "upload_s": upload_s, "device_bytes": info["device_bytes"],
                                  "device_bytes_over_csr": info["device_bytes"] / csr_bytes}
        # the opt-in column-panel copy: every row summed in the reference's
        # order (bit-identical products), at its own speed
        t0 = time.perf_counter()
        built = Zd.add_panels()
        panel_s = time.perf_counter() - t0
        if built:
            ms = time_device(lambda: Zd.spmv(xz, yz, stream=sptr), 200, 20, stream)
            info = Zd.info()
            out[f"zipf_csr_panels_{tag}"] = {"gbs": info["spmv_bytes"] / ms / 1e6, "us": ms * 1e3,
                                             "layout": Zd.layout(), "build_s": panel_s,
                                             "device_bytes": info["device_bytes"]}
        for fmt, conv in (("jad", gpu.to_jagged_diagonal), ("ell", gpu.to_ellpack)):
            H = conv(Zd)
            ms = time_device(lambda: H.spmv(xz, yz, stream=sptr), 40, 5, stream)
            out[f"zipf_{fmt}_{tag}"] = {"gbs": H.info()["spmv_bytes"] / ms / 1e6, "us": ms * 1e3,
                                        "device_bytes": H.info()["device_bytes"]}
            H.close()
        Zd.close()
    return out


def _timed_convert(make, reps=7):
    """Median wall time of a synchronous device conversion (after one
    untimed call), the median device time of its kernels (events around
    them, sk_matrix_build_ms) and the info of the handle it built."""
    import torch
    make().close()
    ts, ds = [], []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = make()
        ts.append(time.perf_counter() - t0)
        ds.append(h.build_ms())
        info = h.info()
        h.close()
    return float(np.median(ts)), float(np.median(ds)), info


def convert_bytes(fmt, n, nnz, vbytes, info, block=None):
    """Algorithmic bytes of one conversion: the CSR read once, the new
    layout written once (ELL with its slot stride and padding)."""
    read = 4 * (n + 1) + nnz * (4 + vbytes)
    if fmt == "ell":
        ld = (n + 31) // 32 * 32 + 96
        return read + ld * info["width"] * (4 + vbytes) + 4 * n
    if fmt == "jad":
        return read + 8 * n + 4 * (info["width"] + 1) + nnz * (4 + vbytes)
    br, bc = block
    nbr = (n + br - 1) // br
    return read + 4 * (nbr + 1) + info["width"] * (4 + br * bc * vbytes)


def convert_cases(grid):
    from sparkit_b200 import matgen
    A = matgen.laplacian_3d_dirichlet(grid)
    V = matgen.vector_laplacian_3d_bsr_csr(grid, seed=1)
    Z = matgen.zipf_random(1_000_000, s=1.5, cap=2048, seed=0)
    # (tag, matrix, format, block, rows of the reference's sample)
    return [("lap3d_ell", A, "ell", None, 1 << 18), ("lap3d_jad", A, "jad", None, 1 << 18),
            ("vec3_bsr33", V, "bsr", (3, 3), 3 << 17), ("zipf_jad", Z, "jad", None, 25_000),
            ("zipf_ell", Z, "ell", None, 25_000)]


def convert_runs(grid):
    """Device-side construction of the sweep's layouts from CSR handles
    (sk_ell_from_csr / sk_jad_from_csr / sk_bsr_from_csr), FP64: the
    synchronous call (allocation, kernels, the scalars read back) and the
    device time of its kernels, as CSR entries converted per second, and
    the algorithmic GB/s of the kernels; beside each, the compiled
    reference's own host conversion on a row sample of the same matrix
    (one core)."""
    from oracle.binding import Reference, reference_available
    from sparkit_b200 import formats, gpu
    peak, _ = measured_peak()
    ref = Reference() if reference_available() else None
    out = {}
    for tag, M, fmt, blk, rows in convert_cases(grid):
        Cd = gpu.Device_matrix(M)
        make = {"ell": lambda: gpu.to_ellpack(Cd), "jad": lambda: gpu.to_jagged_diagonal(Cd),
                "bsr": lambda: gpu.to_block_sparse_row(Cd, *blk)}[fmt]
        secs, dev_ms, info = _timed_convert(make)
        Cd.close()
        n, nnz = M.shape()[0], M.size()
        nbytes = convert_bytes(fmt, n, nnz, 8, info, blk)
        dev_s = dev_ms * 1e-3
        row = {"call_ms": secs * 1e3, "device_ms": dev_ms, "nnz": nnz, "width": info["width"],
               "mnnz_per_s": nnz / secs / 1e6, "device_mnnz_per_s": nnz / dev_s / 1e6,
               "device_gbs": nbytes / dev_s / 1e9, "frac_of_measured_peak": nbytes / dev_s / 1e9 / peak,
               "bytes_model": nbytes}
        if ref is not None:
            rp = M.row_ptr()[: rows + 1].copy()
            S = formats.Compressed_row_matrix((rows, M.shape()[1]), rp, M.col_ind()[: rp[-1]],
                                              M.values()[: rp[-1]])
            rs = ref.convert_seconds(S, fmt, blk or (3, 3))
            row["cpu_reference"] = {"mnnz_per_s": S.size() / rs / 1e6, "s": rs, "cores": 1, "kind": "reference",
                                    "sample": f"rows 0..{rows} ({S.size()} entries)"}
            row["speedup_vs_reference"] = row["mnnz_per_s"] / row["cpu_reference"]["mnnz_per_s"]
        out[tag] = row
    return out


def profile_convert(grid):
    """Each device conversion once, for an ncu launch list."""
    import torch

    from sparkit_b200 import gpu
    torch.cuda.set_device(0)
    for tag, M, fmt, blk, _ in convert_cases(grid):
        Cd = gpu.Device_matrix(M)
        h = {"ell": lambda: gpu.to_ellpack(Cd), "jad": lambda: gpu.to_jagged_diagonal(Cd),
             "bsr": lambda: gpu.to_block_sparse_row(Cd, *blk)}[fmt]()
        h.close()
        Cd.close()
    torch.cuda.synchronize()
    return 0


def eigen_runs(grid):
    """estimate_eigenvalue_bounds (conditioning.hpp:132, two Lanczos passes
    of Krylov dimension 31, up to 10 restarts each) through
    sk_eigenvalue_bounds on the grid^3 and 48^3 Dirichlet Laplacians: wall
    time of the synchronous call (its restart decisions read two scalars
    per Lanczos step back to the host), median of 3 after one warm-up;
    beside it the compiled reference's own estimate on the 48^3 matrix (one
    core)."""
    from oracle.binding import Reference, reference_available
    from sparkit_b200 import gpu, matgen
    out = {}
    for g in (grid, 48):
        A = matgen.laplacian_3d_dirichlet(g)
        Ad = gpu.Device_matrix(A)
        gpu.estimate_eigenvalue_bounds(Ad)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            lo, hi = gpu.estimate_eigenvalue_bounds(Ad)
            ts.append(time.perf_counter() - t0)
        c = 6 * np.cos(np.pi / (g + 1))
        row = {"n": A.shape()[0], "ms": float(np.median(ts)) * 1e3, "lambda_min": lo, "lambda_max": hi,
               "exact": [6 - c, 6 + c]}
        if g == 48 and reference_available():
            R = Reference()
            t0 = time.perf_counter()
            rb = R.eigenvalue_bounds(A)
            rs = time.perf_counter() - t0
            row["cpu_reference"] = {"s": rs, "cores": 1, "kind": "reference", "lambda_min": float(rb[0]),
                                    "lambda_max": float(rb[1])}
            row["speedup_vs_reference"] = rs / (row["ms"] * 1e-3)
        out[f"lap3d_{g}"] = row
        Ad.close()
    return out


def profile_eigen(grid):
    """One sk_eigenvalue_bounds on the grid^3 Laplacian, for an ncu launch list."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    Ad = gpu.Device_matrix(matgen.laplacian_3d_dirichlet(grid))
    gpu.estimate_eigenvalue_bounds(Ad)
    torch.cuda.synchronize()
    return 0


def mm_runs(grid):
    """Matrix Market file -> device CSR handle (sk_matrix_market_read, all
    host cores parsing, the assembly on the device) for the grid^3
    Laplacian written with 17 significant digits: wall time of the call
    (median of 3 after one warm-up, the file in the page cache), text MB/s
    and entries/s; beside it the compiled reference's read_matrix_market +
    to_compressed_row on the file's first 262,144 entry lines (one core)."""
    import tempfile

    from oracle.binding import Reference, reference_available
    from sparkit_b200 import gpu, matgen
    A = matgen.laplacian_3d_dirichlet(grid)
    nnz = A.size()
    out = {"nnz": nnz, "threads": os.cpu_count()}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "lap.mtx")
        Ad = gpu.Device_matrix(A)
        t0 = time.perf_counter()
        gpu.write_matrix_market(Ad, path, precision=17)
        out["write_ms"] = (time.perf_counter() - t0) * 1e3
        Ad.close()
        size = os.path.getsize(path)
        gpu.read_matrix_market(path).close()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            B = gpu.read_matrix_market(path)
            ts.append(time.perf_counter() - t0)
            B.close()
        secs = float(np.median(ts))
        out.update({"file_mb": size / 1e6, "read_ms": secs * 1e3, "mb_per_s": size / secs / 1e6,
                    "mentries_per_s": nnz / secs / 1e6})
        if reference_available():
            sample = 1 << 18
            with open(path, "rb") as f:
                lines = f.read().split(b"\n")
            head = lines[1].split()
            text = b"\n".join([lines[0], b" ".join([head[0], head[1], str(sample).encode()])] +
                               lines[2:2 + sample]) + b"\n"
            rs = Reference().mm_read_seconds(text)
            out["cpu_reference"] = {"s": rs, "mentries_per_s": sample / rs / 1e6, "cores": 1, "kind": "reference",
                                    "sample": f"the first {sample} entry lines of the same file"}
            out["speedup_vs_reference"] = out["mentries_per_s"] / out["cpu_reference"]["mentries_per_s"]
    return out


def krylov_runs():
    """GMRES(30), CGS and BiCGSTAB with a left Jacobi preconditioner on the
    256^2 upwind convection-diffusion problem, MINRES and CG with Jacobi on
    the 48^3 Dirichlet Laplacian, all to 1e-10: wall time of the host-array
    call (b and x copied in and out; median of 3 after one warm-up) beside
    the compiled reference's own solver on the same problem (one core); and
    the device solvers alone on the 1024^2 / 128^3 versions."""
    from oracle.binding import Reference, reference_available
    from sparkit_b200 import gpu, matgen
    ref = Reference() if reference_available() else None

    def spec(n, A, b):
        Ad = gpu.Device_matrix(A)
        J = gpu.jacobi(Ad)
        op = gpu.spmv(Ad)
        maxit = 40000
        return {
            "gmres30": (lambda x: gpu.gmres(b, x, gpu.Gmres_config(1e-10, 30, maxit), op, left=J),
                        lambda: ref.gmres(A, b, np.zeros(n), 1e-10, 30, maxit, left="jacobi")),
            "cgs": (lambda x: gpu.cgs(b, x, gpu.Cgs_config(1e-10, maxit), op, left=J),
                    lambda: ref.cgs(A, b, np.zeros(n), 1e-10, maxit, left="jacobi")),
            "bicgstab": (lambda x: gpu.bicgstab(b, x, gpu.Bicgstab_config(1e-10, maxit), op, J),
                         lambda: ref.bicgstab(A, b, np.zeros(n), 1e-10, maxit, left="jacobi")),
            "minres": (lambda x: gpu.minres(b, x, gpu.Minres_config(1e-10, maxit), op, left=J),
                       lambda: ref.minres(A, b, np.zeros(n), 1e-10, maxit, left="jacobi")),
            "cg": (lambda x: gpu.conjugate_gradient(b, x, gpu.CGConfig(1e-10, maxit, maxit), op, J, gpu.identity),
                   lambda: ref.cg(A, b, np.zeros(n), 1e-10, maxit, maxit, left="jacobi")),
        }, Ad

    def timed(fn, n):
        fn(np.zeros(n))
        ts, s = [], None
        for _ in range(3):
            x = np.zeros(n)
            t0 = time.perf_counter()
            s = fn(x)
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), s, x

    out = {}
    problems = [("convdiff_256sq", matgen.convection_diffusion_2d(256, 256, 1.0, 0.9, 0.5), ("gmres30", "cgs", "bicgstab"), True),
                ("lap3d_48", matgen.laplacian_3d_dirichlet(48), ("minres", "cg"), True),
                ("convdiff_1024sq", matgen.convection_diffusion_2d(1024, 1024, 1.0, 0.9, 0.5), ("gmres30", "cgs", "bicgstab"),
                 False),
                ("lap3d_128", matgen.laplacian_3d_dirichlet(128), ("minres", "cg"), False)]
    from oracle.binding import Oracle
    orc = Oracle()  # the true residual check
    for pname, A, solvers, with_ref in problems:
        n = A.shape()[0]
        b = orc.spmv(A, matgen.uniform_vector(n, seed=2))
        fns, Ad = spec(n, A, b)
        for sname in solvers:
            g, r = fns[sname]
            secs, st, x = timed(g, n)
            rel = float(np.linalg.norm(b - orc.spmv(A, x)) / np.linalg.norm(b))
            row = {"n": n, "ms": secs * 1e3, "iterations": st.computed_iterations, "converged": bool(st.converged),
                   "true_rel_residual": rel, "us_per_iteration": secs * 1e6 / max(st.computed_iterations, 1)}
            if with_ref and ref is not None:
                t0 = time.perf_counter()
                _, rs = r()
                rsec = time.perf_counter() - t0
                row["cpu_reference"] = {"s": rsec, "iterations": rs["computed_iterations"],
                                        "converged": bool(rs["converged"]), "cores": 1, "kind": "reference"}
                row["speedup_vs_reference"] = rsec / secs
            out[f"{pname}/{sname}"] = row
        Ad.close()
    return out


def solver_runs(grid3):
    """Time-to-solution of the solver configurations (wall time of the
    solve call, inputs resident on the device, one warm-up solve first).

    c1: Jacobi-CG, 256^2 Dirichlet 5-point Laplacian, b = A x*, x* ~ U[-1,1]
        seed 0, to 1e-10 -- GPU FP64 vs the reference on one host core.
    c3: 3-D 7-point diffusion, GRF coefficients exp(g) (sigma 2, correlation
        8 cells) on grid3^3, b ~ U[-1,1] seed 0, to a 1e-10 relative residual
        -- plain FP64 Jacobi-CG vs FP32-inner (1e-5) / FP64-refinement."""
    import torch

    from sparkit_b200 import gpu, matgen
    out = {}
    # ---- c1
    A = matgen.laplacian_2d_dirichlet(256)
    n = A.shape()[0]
    Ad = gpu.Device_matrix(A)
    xs = matgen.uniform_vector(n, seed=0)
    b = gpu.multiply(Ad, xs)
    bd = torch.from_numpy(b).cuda()
    J = gpu.jacobi(Ad)
    cfg = gpu.CGConfig(1e-10, 100000, 100000)
    for rep in range(2):
        xd = torch.zeros_like(bd)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s1 = gpu.conjugate_gradient(bd, xd, cfg, gpu.spmv(Ad), J)
        torch.cuda.synchronize()
        t_gpu = time.perf_counter() - t0
    r = b - gpu.multiply(Ad, xd.cpu().numpy())
    c1 = {"gpu_ms": t_gpu * 1e3, "iterations": s1.computed_iterations, "converged": s1.converged,
          "true_rel_residual": float(np.linalg.norm(r) / np.linalg.norm(b))}
    try:
        from oracle.binding import Reference, reference_available
        if reference_available():
            R = Reference()
            t0 = time.perf_counter()
            _, sr = R.cg(A, b, np.zeros(n), 1e-10, 100000, 100000, left="jacobi")
            c1["cpu_reference_ms"] = (time.perf_counter() - t0) * 1e3
            c1["cpu_reference_iterations"] = sr["computed_iterations"]
            c1["cpu_cores"] = 1
    except Exception as e:  # the CPU leg is informational
        c1["cpu_reference_error"] = str(e)[:200]
    out["c1_jacobi_cg_256sq"] = c1
    Ad.close()
    # ---- c3
    G = matgen.diffusion_3d_grf(grid3, sigma=2.0, corr_len=8.0, seed=0)
    n = G.shape()[0]
    Gd = gpu.Device_matrix(G)
    Gd.add_f32_values()
    b = matgen.uniform_vector(n, seed=0)
    bd = torch.from_numpy(b).cuda()
    JG = gpu.jacobi(Gd)
    res = {}
    reps_p, reps_m = [], []
    for rep in range(3):
        xd = torch.zeros_like(bd)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sp = gpu.conjugate_gradient(bd, xd, gpu.CGConfig(1e-10, 10 ** 6, 200000), gpu.spmv(Gd), JG)
        torch.cuda.synchronize()
        tp = time.perf_counter() - t0
        reps_p.append(tp * 1e3)
    tp = min(reps_p[1:]) / 1e3
    rp = float(np.linalg.norm(b - gpu.multiply(Gd, xd.cpu().numpy())) / np.linalg.norm(b))
    res["plain_fp64"] = {"ms": tp * 1e3, "iterations": sp.computed_iterations, "converged": sp.converged,
                         "true_rel_residual": rp}
    variants = (("mixed_fp32_fp64", gpu.Mixed_config(1e-10, 1e-5, 100, 200000)),
                ("mixed_per_step_kernels", gpu.Mixed_config(1e-10, 1e-5, 100, 200000, persistent=False)))
    for name, mcfg in variants:
        reps = []
        for rep in range(3):
            xd = torch.zeros_like(bd)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sm = gpu.mixed_cg(bd, xd, mcfg, gpu.spmv(Gd))
            torch.cuda.synchronize()
            reps.append((time.perf_counter() - t0) * 1e3)
        tm = min(reps[1:]) / 1e3
        rm = float(np.linalg.norm(b - gpu.multiply(Gd, xd.cpu().numpy())) / np.linalg.norm(b))
        res[name] = {"ms": tm * 1e3, "outer": sm.outer_iterations, "inner_iterations": sm.inner_iterations,
                     "converged": sm.converged, "true_rel_residual": rm, "inner_ms": sm.inner_ms,
                     "outer_ms": sm.outer_ms, "setup_ms": sm.setup_ms, "persistent": sm.persistent,
                     "us_per_inner_iteration": sm.inner_ms * 1e3 / max(sm.inner_iterations, 1)}
        reps_m.append({name: reps})
        if name == "mixed_fp32_fp64":
            res["speedup_mixed_vs_plain"] = tp / tm
    res["reps_ms"] = {"plain_fp64": reps_p, "mixed": reps_m, "reported": "best of the repetitions after the first"}
    # the same two solvers on a handle carrying the diagonal copy (one value
    # plane per stencil offset, no column indices, x read contiguously);
    # every product keeps its bits, so the iteration counts are the CSR ones
    JG.close()
    Gd.close()
    Dd = gpu.Device_matrix(G)
    dia = {"built": Dd.add_diagonals()}
    Dd.add_f32_values()
    JD = gpu.jacobi(Dd)
    for name, solve in (("plain_fp64", lambda x: gpu.conjugate_gradient(
                            bd, x, gpu.CGConfig(1e-10, 10 ** 6, 200000), gpu.spmv(Dd), JD)),
                        ("mixed_fp32_fp64", lambda x: gpu.mixed_cg(
                            bd, x, gpu.Mixed_config(1e-10, 1e-5, 100, 200000), gpu.spmv(Dd)))):
        reps = []
        for rep in range(3):
            xd = torch.zeros_like(bd)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sv = solve(xd)
            torch.cuda.synchronize()
            reps.append((time.perf_counter() - t0) * 1e3)
        rel = float(np.linalg.norm(b - gpu.multiply(Dd, xd.cpu().numpy())) / np.linalg.norm(b))
        entry = {"ms": min(reps[1:]), "reps_ms": reps, "converged": sv.converged, "true_rel_residual": rel}
        if name == "plain_fp64":
            entry["iterations"] = sv.computed_iterations
        else:
            entry.update({"outer": sv.outer_iterations, "inner_iterations": sv.inner_iterations,
                          "persistent": sv.persistent, "inner_ms": sv.inner_ms,
                          "us_per_inner_iteration": sv.inner_ms * 1e3 / max(sv.inner_iterations, 1)})
        dia[name] = entry
    dia["speedup_mixed_vs_plain"] = dia["plain_fp64"]["ms"] / dia["mixed_fp32_fp64"]["ms"]
    dia["speedup_mixed_vs_plain_csr"] = res["plain_fp64"]["ms"] / dia["mixed_fp32_fp64"]["ms"]
    res["diagonal_copy"] = dia
    JD.close()
    Dd.close()
    res["n"] = n
    res["nnz"] = G.size()
    out[f"c3_grf_diffusion_{grid3}cubed"] = res
    return out


def learned_runs(train_grid=128, instances=200, cycles=100, eval_grids=(128, 512)):
    """c4: the learned FGMRES preconditioner.  (residual, error) pairs are
    harvested from the plain Jacobi-FGMRES(30) runs (one pair per restart
    cycle) on `instances` seeded convection-diffusion instances of
    train_grid^2 (GRF diffusion sigma 1, divergence-free velocity, cell
    Peclet log-uniform in [1, 100]); the network is trained on the GPU by
    the library's own kernels.  Then FGMRES(30) to a 1e-8 relative residual
    on held-out instances: single-level Jacobi, Chebyshev(8) (bounds from a
    power iteration) and the learned preconditioner; and the two-level forms
    (aggregation coarse correction, 8 x 8 cells per aggregate) with Jacobi
    and with a second network, trained on coarse-corrected pairs, as the
    smoother after the coarse correction.  Times are wall times of the solve call with
    inputs on the device; a solve that does not converge within its cap
    reports its cap time and converged = false.  The two-level forms, which
    converge, are solved three times: `first_ms` is the first solve (it
    also allocates the network's workspace and captures the cycle graphs),
    `ms` the median of the two after it, and their ratio is taken on `ms`."""
    import torch

    from oracle.binding import Oracle
    from sparkit_b200 import gpu, matgen
    O = Oracle()
    out = {}
    m = train_grid
    pairs = gpu.Pairs(m, m, instances * cycles, instances)
    t0 = time.perf_counter()
    for seed in range(instances):
        Am = matgen.convdiff_2d_grf(m, seed=100 + seed)[0]
        Amd = gpu.Device_matrix(Am)
        inst = pairs.add_instance(Amd)
        xs = np.random.default_rng(seed).uniform(-1, 1, m * m) if seed % 2 == 0 else \
            matgen.gaussian_random_field((m, m), 1.0, m / 16, seed=seed).ravel()
        pairs.harvest(inst, Amd, torch.from_numpy(O.spmv(Am, xs)).cuda(), torch.from_numpy(xs).cuda(), 30, cycles)
        Amd.close()
    torch.cuda.synchronize()
    out["harvest"] = {"pairs": len(pairs), "grid": m, "instances": instances, "s": time.perf_counter() - t0}
    net = gpu.Net(seed=1)
    ts = net.train(pairs, gpu.Train_config(steps=2000, batch=8, lr=2e-3, mu=1.0, seed=3))
    h = np.array(ts.loss_history)
    out["train"] = {"steps": 2000, "batch": 8, "ms": ts.ms, "loss_first20": float(h[:20].mean()),
                    "loss_last50": float(h[-50:].mean())}
    pairs.close()
    # The network as the smoother of the two-level form sees coarse-corrected
    # residuals only: a second network is trained on pairs (r - A c, e - c)
    # with c = P Ac^-1 P^T r the coarse correction (aggregates of 8 x 8
    # cells), r and e taken after each restart cycle of FGMRES(30) runs on
    # further 128^2 instances; held-out pairs (10 instances) give its loss.
    net2, out["smoother_train"] = gpu.train_coarse_corrected_smoother(m, instances=200, held=10, cycles=40,
                                                                      steps=8000)

    def mixed_vs_plain(M, Ad, A, b, reps=3):
        """FGMRES(30) to a 1e-10 true residual with M: plain FP64 against FP32
        inner FGMRES(30) (FP64 Hessenberg least-squares) in FP64 refinement;
        best wall time of the repetitions after the first."""
        res = {}
        bh = b.cpu().numpy()
        for name in ("plain_fp64", "mixed_fp32_fp64"):
            ts = []
            for _ in range(reps):
                xd = torch.zeros_like(b)
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                if name == "plain_fp64":
                    s = gpu.fgmres(b, xd, gpu.Fgmres_config(1e-10, 30, 6000), gpu.spmv(Ad), M)
                    its = {"iterations": s.computed_iterations}
                else:
                    s = gpu.mixed_fgmres(b, xd, gpu.Mixed_fgmres_config(1e-10, 1e-4, 30, 50, 6000), gpu.spmv(Ad), M)
                    its = {"outer": s.outer_iterations, "inner_iterations": s.inner_iterations,
                           "inner_ms": s.inner_ms, "outer_ms": s.outer_ms}
                torch.cuda.synchronize()
                ts.append((time.perf_counter() - t1) * 1e3)
            rel = float(np.linalg.norm(bh - O.spmv(A, xd.cpu().numpy())) / np.linalg.norm(bh))
            res[name] = {"ms": min(ts[1:]), "converged": bool(s.converged), "true_rel_residual": rel, **its}
        res["speedup_mixed_vs_plain"] = res["plain_fp64"]["ms"] / res["mixed_fp32_fp64"]["ms"]
        return res

    def run(M, Ad, A, b, maxit, repeat=1):
        """One FGMRES(30) solve to 1e-8; with repeat > 1 the first (cold:
        workspace, tensor maps, cycle graphs) is reported apart and `ms` is
        the median of the repeat - 1 solves after it."""
        ts = []
        for _ in range(repeat):
            xd = torch.zeros_like(b)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            s = gpu.fgmres(b, xd, gpu.Fgmres_config(1e-8, 30, maxit), gpu.spmv(Ad), M)
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t1) * 1e3)
        bh = b.cpu().numpy()
        rel = float(np.linalg.norm(bh - O.spmv(A, xd.cpu().numpy())) / np.linalg.norm(bh))
        out = {"iterations": s.computed_iterations, "converged": bool(s.converged),
               "ms": float(np.median(ts[1:])) if repeat > 1 else ts[0], "true_rel_residual": rel, "cap": maxit}
        if repeat > 1:
            out["first_ms"] = ts[0]
        return out

    def power_max(Ad, n, its=80):
        v = torch.randn(n, dtype=torch.float64, device="cuda")
        w = torch.empty_like(v)
        lam = 0.0
        for _ in range(its):
            v /= v.norm()
            Ad.spmv(v, w)
            lam = float(torch.dot(v, w))
            v, w = w, v
        return lam

    for g in eval_grids:
        A, info = matgen.convdiff_2d_grf(g, seed=777)
        Ad = gpu.Device_matrix(A)
        b = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, g * g)).cuda()
        J = gpu.jacobi(Ad)
        lmax = power_max(Ad, g * g) * 1.05
        L = gpu.learned_preconditioner(Ad, net, g, g)
        big = g >= 512
        r = {"grid": g, "peclet": info["peclet"],
             "jacobi": run(J, Ad, A, b, 10000 if big else 6000),
             "chebyshev8": run(gpu.chebyshev_preconditioner(Ad, lmax * 1e-2, lmax, 8), Ad, A, b,
                               2500 if big else 1500),
             "learned": run(L, Ad, A, b, 3000)}
        agg = 8  # aggregates of 8 x 8 cells: a 16^2 coarse grid at 128^2, 64^2 at 512^2
        r["twolevel_jacobi"] = run(gpu.twolevel(Ad, J, g, g, agg), Ad, A, b, 3000, repeat=3)
        L2 = gpu.learned_preconditioner(Ad, net2, g, g)
        r["twolevel_learned_smoother"] = run(gpu.twolevel(Ad, L2, g, g, agg, coarse_first=True), Ad, A, b, 3000,
                                             repeat=3)
        tj, tl = r["twolevel_jacobi"], r["twolevel_learned_smoother"]
        if tj["converged"] and tl["converged"]:
            r["twolevel_learned_vs_jacobi"] = {"iterations": tj["iterations"] / tl["iterations"],
                                               "time": tj["ms"] / tl["ms"]}
        r["twolevel_aggregates"] = [agg, (g // agg) ** 2]
        if big:
            r["fgmres_to_1e-10_fp64_vs_mixed"] = mixed_vs_plain(gpu.twolevel(Ad, J, g, g, agg), Ad, A, b)
            r["twolevel_learned_single_level_network"] = run(gpu.twolevel(Ad, L, g, g, agg, coarse_first=True),
                                                             Ad, A, b, 3000)
        plain = [r["jacobi"], r["chebyshev8"]]
        lt = r["learned"]
        if lt["converged"]:
            best_plain = min(p["ms"] for p in plain)
            r["learned_speedup_vs_plain"] = {
                "value": best_plain / lt["ms"],
                "lower_bound": not any(p["converged"] for p in plain),
                "note": "plain solves that did not converge count with their cap time"}
        out[f"grid{g}"] = r
    return out


def batched_runs(count=4096, loop_sample=64):
    """c5: `count` SPD systems (2-D 5-point / 3-D 7-point Laplacians plus a
    U[0, 0.5] shift, n log-uniform in [1k, 64k], FP32 CSR) solved to a 1e-10
    FP64 residual in one persistent graph-captured launch with the
    autotuned variant, against a loop of the plain FP64 Jacobi-CG solver
    over a seeded random sample of `loop_sample` systems (scaled to all)."""
    import torch

    from sparkit_b200 import gpu, matgen
    from sparkit_b200.formats import Compressed_row_matrix
    t0 = time.perf_counter()
    offs, rp, ci, v, kinds = matgen.batched_spd_systems(count, seed=0)
    gen_s = time.perf_counter() - t0
    B = gpu.Batch(offs, rp, ci, v)
    n = int(offs[-1])
    bd = torch.from_numpy(matgen.uniform_vector(n, seed=1)).cuda()
    xd = torch.zeros_like(bd)
    g, t, ms = B.autotune(bd, xd, sample=512)
    cfg = gpu.Batch_config(lanes_per_row=g, threads_per_cta=t)
    reps = []
    for rep in range(3):
        xd.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        inner, outer, rel, conv = B.solve(bd, xd, cfg)
        torch.cuda.synchronize()
        reps.append((time.perf_counter() - t0) * 1e3)
    batched_ms = min(reps[1:])
    # the plain per-system loop on a seeded sample
    rng = np.random.default_rng(5)
    sample = np.sort(rng.choice(count, size=loop_sample, replace=False))
    b = bd.cpu().numpy()
    loop_ms, loop_nnz, loop_its = 0.0, 0, 0
    for s in sample:
        a, e = int(offs[s]), int(offs[s + 1])
        A = Compressed_row_matrix((e - a, e - a), rp[a:e + 1] - rp[a], ci[rp[a]:rp[e]] - a,
                                  v[rp[a]:rp[e]].astype(np.float64))
        Ad = gpu.Device_matrix(A)
        J = gpu.jacobi(Ad)
        bs = torch.from_numpy(b[a:e].copy()).cuda()
        for rep in range(2):
            xs = torch.zeros_like(bs)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sp = gpu.conjugate_gradient(bs, xs, gpu.CGConfig(1e-10, 10 ** 6, 100000), gpu.spmv(Ad), J)
            torch.cuda.synchronize()
            tt = (time.perf_counter() - t0) * 1e3
        loop_ms += tt
        loop_nnz += A.size()
        loop_its += sp.computed_iterations
        Ad.close()
    loop_all_ms = loop_ms * count / loop_sample
    return {"systems": count, "rows": n, "nnz": int(rp[-1]), "generate_s": gen_s,
            "autotuned": {"lanes_per_row": g, "threads_per_cta": t, "variant_ms": [round(x, 3) for x in ms]},
            "batched_ms": batched_ms, "reps_ms": reps, "all_converged": bool(conv.all()),
            "max_rel_residual": float(rel.max()), "inner_iterations_total": int(inner.sum()),
            "plain_loop_ms_scaled": loop_all_ms, "plain_loop_sample": int(loop_sample),
            "plain_loop_sample_ms": loop_ms, "speedup_batched_vs_loop": loop_all_ms / batched_ms}


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
        if dt == np.float64:  # the CSR handle through its diagonal copy
            Ad = gpu.Device_matrix(Adt)
            assert Ad.add_diagonals()
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


def profile_learned(grid=512, applies=4):
    """The learned preconditioner's apply on the grid^2 convection-diffusion
    matrix, `applies` times (the network's weights do not change the
    kernels' work), for an ncu launch list or capture."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    A, _ = matgen.convdiff_2d_grf(grid, seed=999)
    Ad = gpu.Device_matrix(A)
    net = gpu.Net(seed=1)
    M = gpu.learned_preconditioner(Ad, net, grid, grid)
    v = torch.from_numpy(np.random.default_rng(0).standard_normal(grid * grid)).cuda()
    z = torch.zeros_like(v)
    for _ in range(applies):
        M.apply(v, z)
    torch.cuda.synchronize()
    return 0


def profile_small_solves():
    """The one-launch FP64 solves, each twice (a warm-up, then the captured
    one): Jacobi-CG on the 256^2 Dirichlet Laplacian (configuration 1),
    Jacobi BiCGSTAB and CGS on the 256^2 upwind convection-diffusion
    problem and Jacobi MINRES on the 48^3 Laplacian, all to 1e-10."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)

    def dev(A, seed):
        Ad = gpu.Device_matrix(A)
        b = torch.empty(A.shape()[0], dtype=torch.float64, device="cuda")
        Ad.spmv(torch.from_numpy(matgen.uniform_vector(A.shape()[0], seed=seed)).cuda(), b)
        return Ad, gpu.jacobi(Ad), b

    Ad, J, b = dev(matgen.laplacian_2d_dirichlet(256), 0)
    for _ in range(2):
        gpu.conjugate_gradient(b, torch.zeros_like(b), gpu.CGConfig(1e-10, 100000, 100000), gpu.spmv(Ad), J)
    Cd, JC, c = dev(matgen.convection_diffusion_2d(256, 256, 1.0, 0.9, 0.5), 2)
    for _ in range(2):
        gpu.bicgstab(c, torch.zeros_like(c), gpu.Bicgstab_config(1e-10, 40000), gpu.spmv(Cd), JC)
    for _ in range(2):
        gpu.cgs(c, torch.zeros_like(c), gpu.Cgs_config(1e-10, 40000), gpu.spmv(Cd), JC)
    Ld, JL, l = dev(matgen.laplacian_3d_dirichlet(48), 2)
    for _ in range(2):
        gpu.minres(l, torch.zeros_like(l), gpu.Minres_config(1e-10, 40000), gpu.spmv(Ld), JL)
    torch.cuda.synchronize()
    return 0


def profile_c4(grid=512, iters=60):
    """Two FGMRES(30) cycles on the configuration-4 matrix with the two-level
    preconditioner (aggregates of 8 x 8 cells), first with a network
    smoother (untrained weights: the kernels' work does not depend on
    them), then with Jacobi, for a per-iteration launch list."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    A, _ = matgen.convdiff_2d_grf(grid, seed=777)
    Ad = gpu.Device_matrix(A)
    b = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, grid * grid)).cuda()
    L = gpu.learned_preconditioner(Ad, gpu.Net(seed=1), grid, grid)
    for M in (gpu.twolevel(Ad, L, grid, grid, 8, coarse_first=True), gpu.twolevel(Ad, gpu.jacobi(Ad), grid, grid, 8)):
        x = torch.zeros_like(b)
        gpu.fgmres(b, x, gpu.Fgmres_config(1e-14, 30, iters), gpu.spmv(Ad), M)
    torch.cuda.synchronize()
    return 0


def profile_batched(count=512):
    """The batched CG (lanes per row 1, 1024 threads per CTA) on the first
    `count` systems of the configuration-5 batch, twice."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    offs, rp, ci, v, kinds = matgen.batched_spd_systems(4096, seed=0)
    e = int(offs[count])
    B = gpu.Batch(offs[:count + 1], rp[:e + 1], ci[:rp[e]], v[:rp[e]])
    bd = torch.from_numpy(matgen.uniform_vector(int(offs[-1]), seed=1)[:e]).cuda()
    cfg = gpu.Batch_config(lanes_per_row=1, threads_per_cta=1024)
    for _ in range(2):
        xd = torch.zeros_like(bd)
        B.solve(bd, xd, cfg)
    torch.cuda.synchronize()
    return 0


def profile_mixed(grid, inner=100, diagonals=False):
    """One outer step of the mixed solver on the GRF diffusion problem with
    `inner` persistent FP32 inner iterations, twice (warm-up, then the
    captured one); with `diagonals`, on a handle carrying its diagonal copy."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    G = matgen.diffusion_3d_grf(grid, sigma=2.0, corr_len=8.0, seed=0)
    Gd = gpu.Device_matrix(G)
    if diagonals:
        assert Gd.add_diagonals()
    Gd.add_f32_values()
    b = torch.from_numpy(matgen.uniform_vector(G.shape()[0], seed=0)).cuda()
    for _ in range(2):
        x = torch.zeros_like(b)
        s = gpu.mixed_cg(b, x, gpu.Mixed_config(1e-10, 1e-5, 1, inner), gpu.spmv(Gd))
    torch.cuda.synchronize()
    assert s.persistent and s.inner_iterations == inner
    return 0


def profile_gmres(grid=1024, iters=40):
    """A short Jacobi-left GMRES(30) on the grid^2 upwind convection-diffusion
    problem (`iters` iterations, too few for the cycle to be captured as a
    CUDA graph), for a capture of the Arnoldi step's kernel."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    A = matgen.convection_diffusion_2d(grid, grid, 1.0, 0.9, 0.5)
    n = A.shape()[0]
    Ad = gpu.Device_matrix(A)
    b = matgen.uniform_vector(n, seed=2)
    s = gpu.gmres(b, np.zeros(n), gpu.Gmres_config(1e-10, 30, iters), gpu.spmv(Ad), left=gpu.jacobi(Ad))
    assert s.computed_iterations == iters
    return 0


def profile_zipf(panels=False):
    """Three CSR FP64 products of matrix B (the split product of skewed
    rows, or with `panels` the column-panel copy), for an ncu capture of one
    launch."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    Z = matgen.zipf_random(1_000_000, s=1.5, cap=2048, seed=0)
    Zd = gpu.Device_matrix(Z)
    if panels:
        assert Zd.add_panels()
    xz = torch.from_numpy(matgen.uniform_vector(Z.shape()[0], seed=3)).cuda()
    yz = torch.empty_like(xz)
    for _ in range(3):
        Zd.spmv(xz, yz)
    torch.cuda.synchronize()
    return 0


def profile_solvers(grid):
    """A short plain FP64 Jacobi-CG (20 iterations) and a short mixed solve
    (one outer step of 20 FP32 iterations with one kernel per step, the
    FP32 counterpart of the FP64 kernels) for per-kernel launch lists."""
    import torch

    from sparkit_b200 import gpu, matgen
    torch.cuda.set_device(0)
    G = matgen.diffusion_3d_grf(grid, sigma=2.0, corr_len=8.0, seed=0)
    Gd = gpu.Device_matrix(G)
    Gd.add_f32_values()
    bd = torch.from_numpy(matgen.uniform_vector(G.shape()[0], seed=0)).cuda()
    xd = torch.zeros_like(bd)
    gpu.conjugate_gradient(bd, xd, gpu.CGConfig(1e-10, 10 ** 6, 20), gpu.spmv(Gd), gpu.jacobi(Gd))
    xd.zero_()
    gpu.mixed_cg(bd, xd, gpu.Mixed_config(1e-10, 1e-5, 1, 20, persistent=False), gpu.spmv(Gd))
    torch.cuda.synchronize()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_small_solves:
        return profile_small_solves()
    if args.profile_batched:
        return profile_batched()
    if args.profile_c4:
        return profile_c4()
    if args.profile_formats:
        return profile_formats(args.grid)
    if args.profile_zipf or args.profile_zipf_panels:
        return profile_zipf(panels=args.profile_zipf_panels)
    if args.profile_convert:
        return profile_convert(args.grid)
    if args.profile_eigen:
        return profile_eigen(args.grid)
    if args.profile_solvers:
        return profile_solvers(args.grid)
    if args.profile_learned:
        return profile_learned()
    if args.profile_mixed:
        return profile_mixed(args.grid)
    if args.profile_mixed_diagonals:
        return profile_mixed(args.grid, diagonals=True)
    if args.profile_gmres:
        return profile_gmres()
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

    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        dev_id = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
    except Exception:
        dev_id = str(dev)
    # the sampler starts before the warm-up so that the GPU does not idle
    # (and drop its memory clock) between the warm-up and the timed steps
    sampler = ClockSampler(dev_id)
    time.sleep(0.3)
    warm = max(args.warmup, 3)
    torch.cuda.synchronize()
    h0 = time.perf_counter()
    for _ in range(warm):
        step()
    host_per_call = (time.perf_counter() - h0) / warm
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    # A bounded device-side delay (torch's clock spin, outside the timed
    # region) lets the host queue the first timed launches ahead of the GPU,
    # so the events time back-to-back kernels rather than Python call gaps.
    gate_s = min(0.25, 1.5 * host_per_call * min(args.steps, 1000))
    torch.cuda._sleep(int(gate_s * 2.0e9))
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
                "kernel": "sell_spmv_kernel<double, EpiStore<double>, 4, false, 8>",
                "bytes_model": "8*nnz + 4*nnz + 4*(n+1) + 8*n (x) + 8*n (y)", "bytes_per_launch": bytes_one}

    extra = {}
    if rank == 0 and world == 1 and not args.no_cpu:
        extra["cpu_baseline"] = cpu_baseline(A, x, bytes_one)
    if rank == 0 and world == 1 and not args.no_sweep:
        Ad.close()
        extra["sweep"] = sweep(stream, args.grid)
    if rank == 0 and world == 1 and not args.no_convert:
        extra["convert"] = convert_runs(args.grid)
    if rank == 0 and world == 1 and not args.no_eigen:
        extra["eigen_bounds"] = eigen_runs(args.grid)
    if rank == 0 and world == 1 and not args.no_mm:
        extra["matrix_market"] = mm_runs(args.grid)
    if rank == 0 and world == 1 and not args.no_solvers:
        extra["solvers"] = solver_runs(args.grid)
        extra["solvers"]["c5_batched"] = batched_runs()
        extra["solvers"]["c4_learned_fgmres"] = learned_runs()
        extra["solvers"]["krylov"] = krylov_runs()

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
