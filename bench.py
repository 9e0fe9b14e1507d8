"""Benchmark: HODLR build + HODLR x dense throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the single-GPU benchmark configuration): n = 32768 points in
[0,1]^2 (seed 1) in Morton order, Matern-3/2 kernel with length 0.1 plus
1e-2 I, HODLR depth 8 (leaf 128), truncation tolerance 1e-8; the built
HODLR times X with 256 columns of N(0,1).  Synthetic data, generated on the
device.  A step is one H X product; the tree (776 MB of factors) and X
(64 MB) exceed the 126 MB L2, so no flush is needed between steps.

value  = matmat throughput in algorithmic bytes, B = 8 W + 16 n k per step
         (W = stored elements), inputs resident in HBM.
e2e    = the same metric through multiply_hodlr_dense with host buffers
         (H2D of X and D2H of Y inside every step).
Printed as one JSON line by rank 0.  With --gpus N > 1 every rank runs an
independent replica (the product does not shard); value sums the replicas'
work over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HODLR build s + matmat GB/s, mixed vs FP64 plain at 1e-8 rel err, 1 B200"
WORKLOAD = "matern2d_n32768"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=None, help="override n (testing only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-n", type=int, default=8192,
                    help="n of the in-run CPU baseline sample (our arm)")
    ap.add_argument("--ref-n", type=int, default=16384,
                    help="n of the reference arm: the largest power of two the unmodified "
                         "reference builds")
    ap.add_argument("--no-side", action="store_true",
                    help="skip the n = 1024 H x and n = 16384 H x H measurements")
    ap.add_argument("--batch", type=int, default=512,
                    help="instances of the uneven-batch measurement (0: skip)")
    ap.add_argument("--no-exp3d", action="store_true",
                    help="skip the n = 65536 3D exponential (learned-rank) workload")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout: float = 5.0):
        """Blocks until the sampler has printed its first line (nvidia-smi
        takes a moment to start) or `timeout` seconds pass."""
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.02)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak_tflops(torch, dev):
    """cuBLAS DGEMM 8192^3 throughput on this GPU (FP64 roofline denominator;
    the driver's peak file carries no FP64 figure)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(5):
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def int8_peak_tops(torch, dev):
    """int8 tensor throughput of cuBLASLt (torch._int_mm, 8192^3) on this GPU,
    the denominator of the mixed path's roofline; falls back to twice the
    measured BF16 figure when the int8 GEMM is unavailable."""
    try:
        a = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device=dev)
        b = torch.randint(-127, 127, (8192, 8192), dtype=torch.int8, device=dev)
        bt = b.t()
        for _ in range(2):
            torch._int_mm(a, bt)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for _ in range(5):
            e0.record()
            torch._int_mm(a, bt)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12, "cuBLASLt int8 GEMM 8192^3 measured in this run"
    except Exception:
        bf16 = measured_peaks().get("bf16_tflops", 1590.0)
        return 2.0 * bf16, "2 x measured BF16 dense peak (int8 GEMM unavailable)"


def run_cpu_baseline(n: int, k: int, steps: int = 3, warmup: int = 1, extra=()):
    cmd = [sys.executable, "-m", "oracle.cpu_baseline", "--n", str(n),
           "--height", str(max(1, (n // 128).bit_length() - 1)), "--k", str(k),
           "--steps", str(steps), "--warmup", str(warmup), *extra]
    try:
        out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=1500)
        line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1]
        return json.loads(line)
    except Exception as e:  # the baseline is reported, never required
        return {"error": str(e)[:200]}


def build_stats(lib):
    """Stage times and counters of the calling thread's latest build."""
    st = (C.c_double * 20)()
    lib.hodlr_b200_build_stats(st, 20)
    return {"library_seconds": st[3], "exact_blocks": int(st[0]),
            "sketched_blocks": int(st[1]), "sketch_rounds": int(st[2]),
            "largest_sketch": int(st[9]), "ms_small_svd": st[10], "ms_rounds": st[11],
            "ms_core_svd": st[12], "ms_finish": st[13], "learned_fallbacks": int(st[14]),
            "ms_features": st[15], "gemm_flops": st[16], "input_elems": st[17],
            "ms_host_setup": st[18], "ms_host_plans": st[19]}


def build_roofline(stats, seconds, storage, peak_tflops, peak_gbs, matrix_free=False):
    """Build against both roofs: its algorithmic bytes (the input read once,
    8 n^2, unless matrix-free, plus the factors written once, 8 W) over the
    wall time against the measured HBM bandwidth, and the FP64 GEMM work it
    issued over the wall time against the FP64 GEMM peak measured in the run."""
    nbytes = (0.0 if matrix_free else 8.0 * stats["input_elems"]) + 8.0 * storage
    tflops = stats["gemm_flops"] / seconds / 1e12
    return {"algorithmic_bytes": nbytes, "GB/s": nbytes / seconds / 1e9,
            "frac_hbm": nbytes / seconds / 1e9 / peak_gbs, "gemm_flops": stats["gemm_flops"],
            "TFLOP/s": tflops, "frac_fp64": tflops / peak_tflops,
            "peaks": "HBM copy bandwidth of the driver's measurement; cuBLAS DGEMM of this run"}


def side_workloads(lib, torch, dev, stream, sh):
    """The two smaller workloads of the hot path, measured beside the main
    one: H x on the n = 1024 Gaussian tree (exp(-r^2 / (2 0.2^2)) + I on
    sorted 1D points, seed 0, depth 3, tol 1e-10), device-resident, against
    the dense product; and H_A H_B on n = 16384 (Gaussian l = 0.1 and
    Matern-3/2 l = 0.2, both + I, sorted 1D points seed 3, depth 7, tol 1e-8),
    its time and its error against A (B X) with the dense kernel matrices
    (X: 16 columns of N(0,1)).  Both trees are built from their points on the
    device."""
    from hmat_lib_b200 import workloads as W
    from hmat_lib_b200.hodlr import DeviceTree
    kinds = {"gaussian": 0, "matern32": 1, "exponential": 2}

    def dense(d_pts, n, kind, length, diag):
        a = torch.empty(n * n, dtype=torch.float64, device=dev)
        assert lib.hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, 1, kinds[kind],
                                                length, diag, C.c_void_p(a.data_ptr()), n,
                                                C.c_void_p(sh)) == 0
        return a.view(n, n)          # row-major view of the symmetric matrix

    out = {}
    with torch.cuda.stream(stream):
        # ---- H x, n = 1024
        w = W.WORKLOADS["gauss1d_n1024"]
        n = w["n"]
        d_pts = torch.from_numpy(W.workload_points("gauss1d_n1024").reshape(-1).copy()).to(dev)
        t = DeviceTree.build_kernel(d_pts.data_ptr(), n, 1, kinds[w["kind"]], w["length"],
                                    w["diag"], w["height"], w["tol"], stream=sh)
        x = torch.randn(n, dtype=torch.float64, device=dev)
        y = torch.zeros_like(x)
        for _ in range(20):
            t.matmat(x.data_ptr(), 1, n, y.data_ptr(), n, stream=sh)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 500
        e0.record(stream)
        for _ in range(reps):
            t.matmat(x.data_ptr(), 1, n, y.data_ptr(), n, stream=sh)
        e1.record(stream)
        stream.synchronize()
        a = dense(d_pts, n, w["kind"], w["length"], w["diag"])
        yd = a @ x
        stream.synchronize()
        info = t.info()
        ms = e0.elapsed_time(e1) / reps
        out["matvec_n1024"] = {
            "us_per_matvec": ms * 1e3, "height": w["height"], "tol": w["tol"],
            "GB_per_s": (8.0 * info["storage"] + 16.0 * n) / (ms * 1e-3) / 1e9,
            "rel_err_vs_dense": (torch.linalg.norm(y - yd) / torch.linalg.norm(yd)).item(),
            "note": "device-resident FP64 H x; launch-latency bound at this size"}
        t.free()
        del a
        # ---- H_A H_B, n = 16384
        n, h, tol = 16384, 7, 1e-8
        pts, ka, kb = W.hxh_pair(n, seed=3)
        d_pts = torch.from_numpy(pts.reshape(-1).copy()).to(dev)
        ta = DeviceTree.build_kernel(d_pts.data_ptr(), n, 1, kinds[ka[0]], ka[1], ka[2], h, tol,
                                     stream=sh)
        tb = DeviceTree.build_kernel(d_pts.data_ptr(), n, 1, kinds[kb[0]], kb[1], kb[2], h, tol,
                                     stream=sh)
        stream.synchronize()
        tc = ta.hxh(tb, tol)                      # warm-up (kernels loaded, pool grown)
        tc.free()
        torch.cuda.synchronize()
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            tc = ta.hxh(tb, tol)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            if len(times) < 3:
                tc.free()
        xk = torch.randn(16, n, dtype=torch.float64, device=dev)     # column-major n x 16
        yc = torch.zeros_like(xk)
        tc.matmat(xk.data_ptr(), 16, n, yc.data_ptr(), n, stream=sh)
        ab = torch.zeros_like(xk)
        tb.matmat(xk.data_ptr(), 16, n, ab.data_ptr(), n, stream=sh)
        yh = torch.zeros_like(xk)
        ta.matmat(ab.data_ptr(), 16, n, yh.data_ptr(), n, stream=sh)
        stream.synchronize()
        da = dense(d_pts, n, *ka)
        db = dense(d_pts, n, *kb)
        yd = (xk @ db) @ da                        # rows of (A (B X))^T; A, B symmetric
        stream.synchronize()
        cinfo = tc.info()
        # the same product with its subtree products on the int8 tensor cores
        lib.hodlr_b200_set_option(b"hxh_precision", 1.0)
        try:
            tm = ta.hxh(tb, tol)                  # warm-up: slices and plans
            tm.free()
            torch.cuda.synchronize()
            times_mx = []
            for _ in range(3):
                t0 = time.perf_counter()
                tm = ta.hxh(tb, tol)
                torch.cuda.synchronize()
                times_mx.append(time.perf_counter() - t0)
                if len(times_mx) < 3:
                    tm.free()
        finally:
            lib.hodlr_b200_set_option(b"hxh_precision", 0.0)
        ym = torch.zeros_like(xk)
        tm.matmat(xk.data_ptr(), 16, n, ym.data_ptr(), n, stream=sh)
        stream.synchronize()
        out["hxh_n16384"] = {
            "seconds": min(times), "height": h, "tol": tol,
            "max_rank_out": cinfo["max_rank"],
            "rel_err_vs_dense": (torch.linalg.norm(yc - yd) / torch.linalg.norm(yd)).item(),
            "rel_err_vs_factors_product": (torch.linalg.norm(yc - yh) / torch.linalg.norm(yh)).item(),
            "mixed_subtree_products": {
                "seconds": min(times_mx),
                "rel_err_vs_dense": (torch.linalg.norm(ym - yd) / torch.linalg.norm(yd)).item(),
                "rel_err_vs_fp64_product": (torch.linalg.norm(ym - yc) /
                                            torch.linalg.norm(yc)).item(),
                "option": "hxh_precision=1"},
            "check": "(H_A H_B) X vs A (B X) with the dense kernel matrices, X n x 16"}
        tm.free()
        tc.free()
        ta.free()
        tb.free()
        del da, db
    torch.cuda.empty_cache()
    return out


def exp3d_workload(lib, torch, dev, stream, steps, warmup, peak64=None):
    """The learned-rank workload: n = 65536 points of [0,1]^3 (seed 4) in
    Morton order, exp(-r / 0.15) + 1e-2 I, depth 9 (leaf 128), tol 1e-8,
    k = 128 right-hand sides.  Both trees are built from the points
    (matrix-free: the 34 GB matrix is never formed), first by the plain
    adaptive range finder, then with sketches sized by the shipped rank model
    (fallback to adaptive growth per block).  Then H X in FP64 and in mixed
    precision, device-resident, and the error of both trees' products
    against the dense FP64 product on 16 of the 128 columns, with the kernel
    matrix generated on the device one block of rows at a time."""
    import numpy as np

    from hmat_lib_b200 import rank_model as RM
    from hmat_lib_b200 import workloads as W
    from hmat_lib_b200.hodlr import DeviceTree
    w = W.WORKLOADS["exp3d_n65536"]
    n, h, tol, k = w["n"], w["height"], w["tol"], w["k"]
    sh = stream.cuda_stream
    pts = W.workload_points("exp3d_n65536")
    d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).to(dev)
    out = {"n": n, "height": h, "tol": tol, "k": k,
           "kernel": "exp(-r/0.15) + 1e-2 I, 3D Morton points seed 4",
           "input": "points only (hodlr_b200_build_kernel_dev)"}

    def build(learned):
        lib.hodlr_b200_set_option(b"learned_ranks", 1.0 if learned else 0.0)
        try:
            with torch.cuda.stream(stream):
                stream.synchronize()
                torch.cuda.nvtx.range_push("build_exp3d_learned" if learned else "build_exp3d")
                t0 = time.perf_counter()
                t = DeviceTree.build_kernel(d_pts.data_ptr(), n, 3, 2, w["length"], w["diag"], h,
                                            tol, stream=sh)
                stream.synchronize()
                sec = time.perf_counter() - t0
                torch.cuda.nvtx.range_pop()
        finally:
            lib.hodlr_b200_set_option(b"learned_ranks", 0.0)
        return t, sec, build_stats(lib)

    RM.load_default()
    tree, plain_s, plain_st = build(False)
    tree_l, learned_s, learned_st = build(True)
    ranks, ranks_l = tree.ranks(), tree_l.ranks()
    info = tree.info()

    def by_depth(r):
        return [int(max(r[2 * ((1 << d) - 1):2 * ((1 << (d + 1)) - 1)])) for d in range(h)]

    x = torch.randn(k, n, dtype=torch.float64, device=dev)        # column-major n x k
    y = torch.zeros_like(x)
    bytes_step = 8.0 * info["storage"] + 16.0 * n * k
    flops_step = 2.0 * k * info["storage"]

    def timed(t, precision):
        for _ in range(max(3, warmup)):
            t.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh, precision=precision)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = max(10, steps)
        e0.record(stream)
        for _ in range(reps):
            t.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh, precision=precision)
        e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / reps
        return {"ms_per_step": ms, "GB/s": bytes_step / (ms * 1e-3) / 1e9,
                "GFLOP/s": flops_step / (ms * 1e-3) / 1e9}

    r64 = timed(tree, 0)
    rmx = timed(tree, 1)
    assert lib.hodlr_b200_check(tree.h, C.c_void_p(sh)) == 0, lib.hodlr_b200_last_error()
    # dense product on 16 columns: (A X)[:, :16], A generated 2048 columns at
    # a time (A is symmetric, so a column block is the transposed row block)
    cols, rb = 16, 2048
    xs = x[:cols].contiguous()                      # row c = column c of X
    yd = torch.zeros(cols, n, dtype=torch.float64, device=dev)
    a_blk = torch.empty(n * rb, dtype=torch.float64, device=dev)
    with torch.cuda.stream(stream):
        for r0 in range(0, n, rb):
            assert lib.hodlr_b200_kernel_block_dev(C.c_void_p(d_pts.data_ptr()), n, 3, 2,
                                                   w["length"], w["diag"], 0, r0, n, rb,
                                                   C.c_void_p(a_blk.data_ptr()), n,
                                                   C.c_void_p(sh)) == 0
            blk = a_blk.view(rb, n)                 # blk[j, i] = A[i, r0 + j]
            yd[:, r0:r0 + rb] = xs @ blk.t()        # (A X)[r0 + j, c]
        stream.synchronize()
    del a_blk
    errs = {}
    for name, (t, prec) in (("plain_fp64", (tree, 0)), ("plain_mixed", (tree, 1)),
                            ("learned_fp64", (tree_l, 0)), ("learned_mixed", (tree_l, 1))):
        yy = torch.zeros(k, n, dtype=torch.float64, device=dev)
        t.matmat(x.data_ptr(), k, n, yy.data_ptr(), n, stream=sh, precision=prec)
        stream.synchronize()
        errs[name] = (torch.linalg.norm(yy[:cols] - yd) / torch.linalg.norm(yd)).item()
    tree_l.free()

    # dense input (the 34 GB matrix generated on the device, as hmat_lib's
    # dense_to_tree_hodlr takes it): the plain FP64 build, and the learned build
    # with its sketch products on the int8 tensor cores
    dense = {}
    a = torch.empty(n * n, dtype=torch.float64, device=dev)
    assert lib.hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, 3, 2, w["length"],
                                            w["diag"], C.c_void_p(a.data_ptr()), n,
                                            C.c_void_p(sh)) == 0
    stream.synchronize()
    for name, opts in (("plain_fp64", {}),
                       ("learned_mixed", {b"learned_ranks": 1.0, b"build_precision": 1.0,
                                          b"kernel_length": w["length"]})):
        for key, v in opts.items():
            lib.hodlr_b200_set_option(key, v)
        try:
            with torch.cuda.stream(stream):
                stream.synchronize()
                torch.cuda.nvtx.range_push("build_exp3d_dense_" + name)
                t0 = time.perf_counter()
                td = DeviceTree.build(a.data_ptr(), n, n, h, tol, stream=sh)
                stream.synchronize()
                sec = time.perf_counter() - t0
                torch.cuda.nvtx.range_pop()
        finally:
            for key in opts:
                lib.hodlr_b200_set_option(key, 0.0)
        st = build_stats(lib)
        yy = torch.zeros(k, n, dtype=torch.float64, device=dev)
        td.matmat(x.data_ptr(), k, n, yy.data_ptr(), n, stream=sh)
        stream.synchronize()
        dense[name] = dict(seconds=sec, max_rank_diff_vs_matrix_free=int(np.max(np.abs(
                               td.ranks() - ranks))),
                           rel_err_vs_dense=(torch.linalg.norm(yy[:cols] - yd) /
                                             torch.linalg.norm(yd)).item(), **st)
        td.free()
        del yy
    del a
    torch.cuda.empty_cache()
    dense["speedup_learned_mixed_vs_plain_fp64"] = (dense["plain_fp64"]["seconds"] /
                                                    dense["learned_mixed"]["seconds"])
    out.update({
        "build": {"plain": dict(seconds=plain_s, **plain_st),
                  "learned": dict(seconds=learned_s, **learned_st,
                                  max_rank_diff_vs_plain=int(np.max(np.abs(ranks_l - ranks)))),
                  "speedup_learned_vs_plain": plain_s / learned_s,
                  "roofline_plain": (build_roofline(plain_st, plain_s, info["storage"], peak64,
                                                    measured_peaks().get("hbm_gbs", 6650.0),
                                                    matrix_free=True) if peak64 else None)},
        "ranks_by_depth": by_depth(ranks), "ranks_by_depth_learned": by_depth(ranks_l),
        "factor_bytes": 8 * info["storage"], "max_rank": info["max_rank"],
        "matmat": {"fp64": r64, "mixed": rmx, "bytes_per_step": bytes_step,
                   "speedup_mixed_vs_fp64": r64["ms_per_step"] / rmx["ms_per_step"]},
        "rel_err_vs_dense": errs,
        "build_dense_input": dense,
        "check": "H X vs A X on 16 of the 128 columns, A generated on the device"})
    tree.free()
    del x, y, yd
    torch.cuda.empty_cache()
    return out


def uneven_batch_bench(count, steps, warmup, lib, torch, dev, stream, pg=None, rank=0, world=1):
    """The uneven batch: `count` HODLRs (n in {1024, 2048, 4096, 8192},
    exponential kernel on sorted 1D points, leaf 128, tol 1e-8), each times a
    dense block of 16-128 columns.  Times one step (all instances) three ways:
    one FP64 product call per tree, the batched FP64 call and the batched
    mixed-precision call (one launch per phase, graph replay).  With several
    ranks the instances are partitioned across them (no collective on the
    data path); a step's time is the slowest rank's."""
    import numpy as np

    from hmat_lib_b200 import multi
    from hmat_lib_b200 import workloads as W
    from hmat_lib_b200.hodlr import DeviceTree, batched_tuning, matmat_batched
    sh = stream.cuda_stream
    everything = W.uneven_batch(count, seed=2)
    inst = [everything[i] for i in multi.partition(count, rank, world)]
    nmax = max(it["n"] for it in inst)
    trees, xs, ys, ks, ns = [], [], [], [], []
    build_s = 0.0
    with torch.cuda.stream(stream):
        a = torch.empty(nmax * nmax, dtype=torch.float64, device=dev)
        gen = torch.Generator(device=dev)
        gen.manual_seed(2)
        for it in inst:
            n, k = it["n"], it["k"]
            d_pts = torch.from_numpy(np.ascontiguousarray(it["points"][:, 0])).to(dev)
            r = lib.hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, 1, 2,
                                                 it["length"], 0.0, C.c_void_p(a.data_ptr()), n,
                                                 C.c_void_p(sh))
            assert r == 0
            stream.synchronize()
            t0 = time.perf_counter()
            trees.append(DeviceTree.build(a.data_ptr(), n, n, it["height"], it["tol"], stream=sh))
            build_s += time.perf_counter() - t0
            xs.append(torch.randn(k, n, dtype=torch.float64, device=dev, generator=gen))
            ys.append(torch.zeros(k, n, dtype=torch.float64, device=dev))
            ks.append(k)
            ns.append(n)
        del a
    torch.cuda.empty_cache()
    # the same trees built in batches (hodlr_b200_build_batched_dev): groups of
    # consecutive trees whose dense inputs take at most 40 GB together, each
    # group's inputs generated first, then one batched build per group (the
    # timed part); ranks compared with the per-tree builds
    batched_s, rank_mismatch = 0.0, 0
    groups, cur, cur_b = [], [], 0
    for i, it in enumerate(inst):
        b = 8 * it["n"] * it["n"]
        if cur and cur_b + b > 40e9:
            groups.append(cur)
            cur, cur_b = [], 0
        cur.append(i)
        cur_b += b
    if cur:
        groups.append(cur)
    group = max(len(g) for g in groups)
    batched_stages = {}
    with torch.cuda.stream(stream):
        for gi in groups:
            g0 = gi[0]
            grp = [inst[i] for i in gi]
            mats = []
            for it in grp:
                n = it["n"]
                d_pts = torch.from_numpy(np.ascontiguousarray(it["points"][:, 0])).to(dev)
                m = torch.empty(n * n, dtype=torch.float64, device=dev)
                assert lib.hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, 1, 2,
                                                        it["length"], 0.0,
                                                        C.c_void_p(m.data_ptr()), n,
                                                        C.c_void_p(sh)) == 0
                mats.append(m)
            stream.synchronize()
            t0 = time.perf_counter()
            bt = DeviceTree.build_batched([m.data_ptr() for m in mats], [it["n"] for it in grp],
                                          [it["n"] for it in grp], [it["height"] for it in grp],
                                          1e-8, stream=sh)
            stream.synchronize()
            batched_s += time.perf_counter() - t0
            bst = build_stats(lib)
            for key in ("ms_small_svd", "ms_rounds", "ms_core_svd", "ms_finish", "ms_host_setup",
                        "ms_host_plans", "library_seconds"):
                batched_stages[key] = batched_stages.get(key, 0.0) + bst[key]
            batched_stages["sketch_rounds"] = max(batched_stages.get("sketch_rounds", 0),
                                                  bst["sketch_rounds"])
            for j, t in enumerate(bt):
                rank_mismatch += int(np.any(t.ranks() != trees[g0 + j].ranks()))
                t.free()
            del mats
            torch.cuda.empty_cache()
    batched_s = multi.max_over_ranks(batched_s, pg, dev)
    storage = multi.sum_over_ranks(sum(t.info()["storage"] for t in trees), pg, dev)
    bytes_step = multi.sum_over_ranks(8.0 * sum(t.info()["storage"] for t in trees) +
                                      sum(16.0 * n * k for n, k in zip(ns, ks)), pg, dev)
    build_s = multi.max_over_ranks(build_s, pg, dev)
    xp, yp = [x.data_ptr() for x in xs], [y.data_ptr() for y in ys]

    def loop_step():
        for t, x, y, n, k in zip(trees, xs, ys, ns, ks):
            t.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh)

    def batched_step(precision, out):
        matmat_batched(trees, xp, ks, ns, out, ns, precision=precision, stream=sh)

    def timed(fn, nsteps):
        for _ in range(warmup):
            fn()
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = lib.hodlr_b200_kernel_launches()
        e0.record(stream)
        for _ in range(nsteps):
            fn()
        e1.record(stream)
        stream.synchronize()
        ms = multi.max_over_ranks(e0.elapsed_time(e1) / nsteps, pg, dev)
        return {"ms_per_step": ms, "GB/s": bytes_step / (ms * 1e-3) / 1e9,
                "gpu_launches_per_step": (lib.hodlr_b200_kernel_launches() - l0) / nsteps}

    nsteps = max(5, steps // 8)
    loop = timed(loop_step, max(3, nsteps // 4))
    y64 = [y.clone() for y in ys]
    b64 = timed(lambda: batched_step(0, yp), nsteps)
    tuning = batched_tuning()
    y64b = [y.clone() for y in ys]
    ymx = [torch.zeros_like(y) for y in ys]
    bmx = timed(lambda: batched_step(1, [y.data_ptr() for y in ymx]), nsteps)
    assert lib.hodlr_b200_batched_check() == 0, lib.hodlr_b200_last_error()
    num = multi.sum_over_ranks(sum(float(torch.linalg.norm(m - f) ** 2)
                                   for m, f in zip(ymx, y64b)), pg, dev)
    den = multi.sum_over_ranks(sum(float(torch.linalg.norm(f) ** 2) for f in y64b), pg, dev)
    numb = multi.sum_over_ranks(sum(float(torch.linalg.norm(b - f) ** 2)
                                    for b, f in zip(y64b, y64)), pg, dev)
    out = {"instances": count, "ranks": world, "partition": "instance i on rank i mod ranks",
           "sizes": sorted(set(ns)), "k_range": [min(ks), max(ks)],
           "kernel": "exp(-|x-y|/l), l ~ U[0.05,0.5], sorted 1D points, seed 2",
           "build_s_total": build_s,
           "build_batched": {"seconds": batched_s, "calls": len(groups), "largest_call": group,
                             "grouping": "consecutive trees, dense inputs <= 40 GB per call",
                             "stages_summed_over_calls": batched_stages,
                             "speedup_vs_per_tree": build_s / max(batched_s, 1e-9),
                             "trees_with_other_ranks": rank_mismatch,
                             "entry": "hodlr_b200_build_batched_dev"},
           "storage_doubles": storage, "bytes_per_step": bytes_step,
           "loop_fp64": loop, "batched_fp64": b64, "batched_mixed": bmx,
           "speedup_batched_mixed_vs_loop_fp64": loop["ms_per_step"] / bmx["ms_per_step"],
           "rel_err_batched_fp64_vs_loop": (numb / den) ** 0.5,
           "rel_err_mixed_vs_fp64": (num / den) ** 0.5, "tuning": tuning}
    lib.hodlr_b200_batched_release()
    for t in trees:
        t.free()
    return out


def reference_arm(args, rank):
    """The reference's own CPU implementation (unmodified hmat_lib built in
    oracle/_ref) on this box's host cores, same metric and unit."""
    if rank != 0:
        return
    # every step is one multiply_hodlr_dense of the reference's own build of
    # the workload's kernel family at n = 16384 (the largest power of two its
    # constructor reaches; its factors, about 170 MB, exceed the host caches
    # like the n = 32768 tree's); building it takes the reference a few
    # minutes, the K steps about a tenth of a second each
    steps, warmup = max(1, args.steps), max(0, args.warmup)
    res = run_cpu_baseline(args.ref_n, 256, steps, warmup, extra=("--batch-sample", "2"))
    if "error" in res:
        print(json.dumps({"impl": "reference", "unavailable": res["error"]}))
        return
    nthreads = res["threads"]
    sample = (f"hmat_lib multiply_hodlr_dense, k=256, on its own build of the same kernel "
              f"family at n={res['n']} (depth {res['height']}); the reference constructor "
              f"overflows int at n=32768 (src/constructors.c:676)")
    value = res["matmat_gbs"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GB/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup,
        "ms_per_step": res["matmat_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": WORKLOAD, "n": res["n"],
                                        "height": res["height"], "k": 256, "tol": 1e-8},
        "build_s": res["build_s"],
        "build_s_extrapolated_n32768": res["build_s"] * (32768 / res["n"]) ** 3,
        "cpu_baseline": {"value": value, "unit": "GB/s", "cores": nthreads,
                         "kind": "reference", "sample": sample, "cpu": res.get("cpu")},
        "matvec_n1024_us": res.get("matvec_n1024_us"), "hxh_n4096_s": res.get("hxh_n4096_s"),
        "batch_sample": res.get("batch_sample"),
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import numpy as np
    import torch

    from hmat_lib_b200 import abi
    from hmat_lib_b200 import workloads as W
    from hmat_lib_b200.hodlr import DeviceTree, Tree, lib as hlib

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=dev)
        pg = dist
    lib = hlib()
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream

    w = W.WORKLOADS[WORKLOAD]
    n = args.n or w["n"]
    k, h, tol = w["k"], w["height"] if args.n is None else max(1, (n // 128).bit_length() - 1), w["tol"]

    # ---- input: kernel matrix generated on the device ---------------------------
    pts = W.workload_points(WORKLOAD, n)
    d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).to(dev)
    kind = {"gaussian": 0, "matern32": 1, "exponential": 2}[w["kind"]]

    def make_matrix():
        a = torch.empty(n * n, dtype=torch.float64, device=dev)
        r = lib.hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, pts.shape[1], kind,
                                             w["length"], w["diag"], C.c_void_p(a.data_ptr()), n,
                                             C.c_void_p(sh))
        assert r == 0
        return a

    # ---- build (FP64 plain) -------------------------------------------------------
    with torch.cuda.stream(stream):
        a = make_matrix()
        # untimed warm-up build of the same matrix: loads the kernels and
        # grows the stream-ordered pool to the build's peak scratch (kept
        # mapped, option pool_keep); reported as the first-build time
        t0 = time.perf_counter()
        DeviceTree.build(a.data_ptr(), n, n, h, tol, stream=sh).free()
        stream.synchronize()
        build_s_first = time.perf_counter() - t0
        torch.cuda.nvtx.range_push("build_plain")
        t0 = time.perf_counter()
        tree = DeviceTree.build(a.data_ptr(), n, n, h, tol, stream=sh)
        stream.synchronize()
        build_s = time.perf_counter() - t0
        torch.cuda.nvtx.range_pop()
    info = tree.info()
    ranks = tree.ranks()
    plain_stats = build_stats(lib)

    # ---- matrix-free build: the same tree from the points, no n x n matrix ------------
    with torch.cuda.stream(stream):
        stream.synchronize()
        torch.cuda.nvtx.range_push("build_matrix_free")
        t0 = time.perf_counter()
        tree_mf = DeviceTree.build_kernel(d_pts.data_ptr(), n, pts.shape[1], kind, w["length"],
                                          w["diag"], h, tol, stream=sh)
        stream.synchronize()
        build_s_mf = time.perf_counter() - t0
        torch.cuda.nvtx.range_pop()
    mf_stats = build_stats(lib)
    mf_rank_diff = int(np.max(np.abs(tree_mf.ranks() - ranks)))
    tree_mf.free()

    # ---- learned build: sketches sized in one shot by the shipped rank model ------
    from hmat_lib_b200 import rank_model as RM
    RM.load_default()
    lib.hodlr_b200_set_option(b"learned_ranks", 1.0)
    lib.hodlr_b200_set_option(b"kernel_length", w["length"])
    try:
        with torch.cuda.stream(stream):
            # untimed warm-up, as for the plain build: the first learned build
            # in the process also loads the feature and predictor kernels
            stream.synchronize()
            t0 = time.perf_counter()
            DeviceTree.build(a.data_ptr(), n, n, h, tol, stream=sh).free()
            stream.synchronize()
            build_s_learned_first = time.perf_counter() - t0
            torch.cuda.nvtx.range_push("build_learned")
            t0 = time.perf_counter()
            tree_l = DeviceTree.build(a.data_ptr(), n, n, h, tol, stream=sh)
            stream.synchronize()
            build_s_learned = time.perf_counter() - t0
            torch.cuda.nvtx.range_pop()
    finally:
        lib.hodlr_b200_set_option(b"learned_ranks", 0.0)
        lib.hodlr_b200_set_option(b"kernel_length", 0.0)
    learned_stats = build_stats(lib)
    ranks_l = tree_l.ranks()

    # ---- learned + mixed build: one-shot sketches and their products (Y = A Omega,
    # B^T = A^T Q) on the int8 tensor cores (option build_precision) ----------------
    lib.hodlr_b200_set_option(b"learned_ranks", 1.0)
    lib.hodlr_b200_set_option(b"kernel_length", w["length"])
    lib.hodlr_b200_set_option(b"build_precision", 1.0)
    try:
        with torch.cuda.stream(stream):
            stream.synchronize()
            DeviceTree.build(a.data_ptr(), n, n, h, tol, stream=sh).free()   # warm-up
            stream.synchronize()
            torch.cuda.nvtx.range_push("build_learned_mixed")
            t0 = time.perf_counter()
            tree_lm = DeviceTree.build(a.data_ptr(), n, n, h, tol, stream=sh)
            stream.synchronize()
            build_s_lm = time.perf_counter() - t0
            torch.cuda.nvtx.range_pop()
    finally:
        lib.hodlr_b200_set_option(b"learned_ranks", 0.0)
        lib.hodlr_b200_set_option(b"kernel_length", 0.0)
        lib.hodlr_b200_set_option(b"build_precision", 0.0)
    lm_stats = build_stats(lib)
    ranks_lm = tree_lm.ranks()

    # ---- accuracy against the dense FP64 product (checker: cuBLAS on A) ------------
    x = torch.randn(k, n, dtype=torch.float64, device=dev)      # column-major n x k
    y = torch.zeros(k, n, dtype=torch.float64, device=dev)
    tree.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh)
    stream.synchronize()
    a_mat = a.view(n, n)          # row-major view of column-major A = A^T
    y_dense = (x @ a_mat)         # (k x n) = (A X)^T in column-major terms
    rel_err = (torch.linalg.norm(y - y_dense) / torch.linalg.norm(y_dense)).item()
    y_l = torch.zeros(k, n, dtype=torch.float64, device=dev)
    tree_l.matmat(x.data_ptr(), k, n, y_l.data_ptr(), n, stream=sh)
    stream.synchronize()
    rel_err_learned = (torch.linalg.norm(y_l - y_dense) / torch.linalg.norm(y_dense)).item()
    y_l.zero_()
    tree_lm.matmat(x.data_ptr(), k, n, y_l.data_ptr(), n, stream=sh)
    stream.synchronize()
    rel_err_lm = (torch.linalg.norm(y_l - y_dense) / torch.linalg.norm(y_dense)).item()
    del y_l
    tree_l.free()
    tree_lm.free()
    del a, a_mat, y_dense
    torch.cuda.empty_cache()

    # ---- mixed-precision accuracy (same X) ---------------------------------------------
    y_mx = torch.zeros(k, n, dtype=torch.float64, device=dev)
    tree.matmat(x.data_ptr(), k, n, y_mx.data_ptr(), n, stream=sh, precision=1)
    stream.synchronize()
    assert lib.hodlr_b200_check(tree.h, C.c_void_p(sh)) == 0, lib.hodlr_b200_last_error()
    rel_err_mixed_vs_fp64 = (torch.linalg.norm(y_mx - y) / torch.linalg.norm(y)).item()
    del y_mx

    # ---- timed device-resident products -------------------------------------------
    storage = info["storage"]
    bytes_step = 8.0 * storage + 16.0 * n * k
    flops_step = 2.0 * k * storage

    def timed(precision, steps, tag):
        for _ in range(args.warmup):
            tree.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh, precision=precision)
        stream.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        lib.hodlr_b200_set_option(b"record_phase_times", 1.0)
        lib.hodlr_b200_phase_times(None, 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            # The timed region can be shorter than the sampler's 200 ms
            # interval, so the clocks are sampled over a run of the same
            # product of at least one second right before it, and during it.
            clk.wait_first()
            t_pre = time.perf_counter()
            while time.perf_counter() - t_pre < 1.0:
                for _ in range(10):
                    tree.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh,
                                precision=precision)
                stream.synchronize()
            lib.hodlr_b200_phase_times(None, 0)
            launches0 = lib.hodlr_b200_kernel_launches()
            torch.cuda.nvtx.range_push(tag)     # lets ncu select the timed launches
            e0.record(stream)
            for _ in range(steps):
                tree.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh, precision=precision)
            e1.record(stream)
            stream.synchronize()
            torch.cuda.nvtx.range_pop()
        launches = lib.hodlr_b200_kernel_launches() - launches0
        lib.hodlr_b200_set_option(b"record_phase_times", 0.0)
        pt = (C.c_double * 5)()
        lib.hodlr_b200_phase_times(pt, 5)
        ms_total = e0.elapsed_time(e1)
        if pg:
            t = torch.tensor([ms_total], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms_total = t.item()
            pg.barrier()
        torch.cuda.synchronize()
        clocks = clk.summary()
        clocks["window"] = ("nvidia-smi every 200 ms over >= 1 s of the same product run "
                            "immediately before the timed region, and during it")
        return dict(ms=ms_total / steps, launches=int(launches), clocks=clocks,
                    p1=pt[0] / max(pt[2], 1), p2=pt[1] / max(pt[2], 1),
                    k1=pt[3] / max(pt[2], 1), k2=pt[4] / max(pt[2], 1))

    r64 = timed(0, max(20, args.steps // 4), "matmat")
    rmx = timed(1, args.steps, "matmat_mixed")
    assert lib.hodlr_b200_check(tree.h, C.c_void_p(sh)) == 0, lib.hodlr_b200_last_error()
    value = bytes_step * world / (rmx["ms"] * 1e-3) / 1e9
    value_fp64 = bytes_step * world / (r64["ms"] * 1e-3) / 1e9
    ms_step = rmx["ms"]

    # ---- direct solve: factorise once, then X = A^-1 B through the factor ---------------
    tree.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh)     # B = A x (FP64)
    stream.synchronize()
    torch.cuda.nvtx.range_push("factorize")
    t0 = time.perf_counter()
    fac = tree.factorize(stream=sh)
    factor_s = time.perf_counter() - t0
    torch.cuda.nvtx.range_pop()
    xs = torch.zeros_like(x)
    fac.solve(y.data_ptr(), k, n, xs.data_ptr(), n, stream=sh)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    solve_reps = 5
    torch.cuda.nvtx.range_push("solve")
    e0.record(stream)
    for _ in range(solve_reps):
        fac.solve(y.data_ptr(), k, n, xs.data_ptr(), n, stream=sh)
    e1.record(stream)
    stream.synchronize()
    torch.cuda.nvtx.range_pop()
    solve_ms = e0.elapsed_time(e1) / solve_reps
    r_solve = torch.zeros_like(y)
    tree.matmat(xs.data_ptr(), k, n, r_solve.data_ptr(), n, stream=sh)
    stream.synchronize()
    solve_info = {"factorize_s": factor_s, "ms_per_solve": solve_ms, "rhs": k,
                  "residual": (torch.linalg.norm(r_solve - y) / torch.linalg.norm(y)).item(),
                  "rel_err_vs_x": (torch.linalg.norm(xs - x) / torch.linalg.norm(x)).item()}
    fac.free()
    del xs, r_solve

    # ---- the smaller workloads: H x at n = 1024, H x H at n = 16384 -----------------
    side = side_workloads(lib, torch, dev, stream, sh) if not args.no_side else {}

    # ---- e2e through the C-ABI with host buffers ------------------------------------
    host_tree = tree.to_host()
    xh = torch.randn(k, n, dtype=torch.float64).pin_memory()
    yh = torch.zeros(k, n, dtype=torch.float64).pin_memory()
    ierr = C.c_int(0)
    xp = C.cast(C.c_void_p(xh.data_ptr()), abi.DP)
    yp = C.cast(C.c_void_p(yh.data_ptr()), abi.DP)

    def e2e_time(precision):
        lib.hodlr_b200_set_option(b"matmat_precision", float(precision))
        for _ in range(max(1, args.warmup)):
            lib.multiply_hodlr_dense(host_tree.tp, xp, k, n, yp, n, C.byref(ierr))
        assert ierr.value == 0
        steps = max(5, args.steps // 10)
        t0 = time.perf_counter()
        for _ in range(steps):
            lib.multiply_hodlr_dense(host_tree.tp, xp, k, n, yp, n, C.byref(ierr))
        sec = (time.perf_counter() - t0) / steps
        lib.hodlr_b200_set_option(b"matmat_precision", 0.0)
        if pg:
            t = torch.tensor([sec], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            sec = t.item()
        return sec

    e2e_s_fp64 = e2e_time(0)
    e2e_s = e2e_time(1)
    e2e = bytes_step * world / e2e_s / 1e9

    exp3d = None
    if not args.no_exp3d:
        # reported, never required: a failure here is recorded in the line
        try:
            exp3d = exp3d_workload(lib, torch, dev, stream, args.steps, args.warmup,
                                   fp64_peak_tflops(torch, dev))
        except Exception as e:
            exp3d = {"error": str(e)[:300]}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()

    batch = None
    if args.batch > 0:
        batch = uneven_batch_bench(args.batch, args.steps, args.warmup, lib, torch, dev, stream,
                                   pg, rank, world)

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return

    # ---- roofline of the dominant kernel ---------------------------------------------
    # Per-phase algorithmic work from the block ranks (halving geometry: every
    # block at depth d is n / 2^(d+1) square).  Phase 1 reads V and X
    # (2 k sum s_b n_b flops); phase 2 reads the leaves, U and X and writes Y
    # (2 k (sum m_leaf^2 + sum s_b m_b) flops).  The mixed path runs every such
    # multiply-add as S(S+1)/2 = 21 int8 slice products on the tensor cores.
    sn = sum(int(ranks[b]) * (n >> ((b // 2 + 1).bit_length())) for b in range(len(ranks)))
    n_leaf = 1 << h
    leaves_el = n_leaf * (n // n_leaf) ** 2
    el = {"phase1": sn, "phase2": leaves_el + sn}
    slice_products = 21
    # int8 operand bytes the mixed kernels must move per phase (6 slices per
    # value, tiles padded as the kernels lay them out), plus the FP64 W / Y
    # written: the algorithmic bytes that the measured DRAM traffic is set
    # against
    def _cdiv(a_, b_):
        return -(-a_ // b_)
    op1 = 6.0 * n * _cdiv(k, 128) * 128
    op2 = 6.0 * (leaves_el + n * _cdiv(k, 64) * 64) + 8.0 * n * k
    for b, s_b in enumerate(int(v) for v in ranks):
        if s_b == 0:
            continue
        nb = n >> ((b // 2 + 1).bit_length())
        ntn = _cdiv(s_b, 64)
        nw = _cdiv(_cdiv(s_b, ntn), 16) * 16
        op1 += 6.0 * ntn * nw * nb + 8.0 * s_b * k
        op2 += 6.0 * nb * _cdiv(s_b, 32) * 32 + 6.0 * _cdiv(s_b, 32) * 32 * _cdiv(k, 64) * 64
    int8_bytes = {"phase1": op1, "phase2": op2}
    # DRAM bytes (read + write) per launch / int8 operand bytes, measured by
    # ncu on the n = 16384 instance of this workload family (a capture of the
    # n = 32768 launch does not fit the profiler's size limit); applied to
    # the operand bytes at this n
    traffic_ratio_i8 = {"phase1": 0.89, "phase2": 0.90}
    peak_i8, peak_src = int8_peak_tops(torch, dev)
    peak64 = fp64_peak_tflops(torch, dev)
    # the dominant kernel: the int8 GEMM launch of the phase whose launch
    # takes longer, timed alone (events on the launching stream just around
    # it); the phase time adds the slicing kernels before it
    dom = "phase1" if rmx["k1"] >= rmx["k2"] else "phase2"
    dom_ms = rmx["k1"] if dom == "phase1" else rmx["k2"]
    dom_phase_ms = rmx["p1"] if dom == "phase1" else rmx["p2"]
    achieved = slice_products * 2.0 * k * el[dom] / (dom_ms * 1e-3) / 1e12
    achieved_phase = slice_products * 2.0 * k * el[dom] / (dom_phase_ms * 1e-3) / 1e12
    dom64 = "phase1" if r64["p1"] >= r64["p2"] else "phase2"
    dom64_ms = r64["p1"] if dom64 == "phase1" else r64["p2"]
    achieved64 = 2.0 * k * el[dom64] / (dom64_ms * 1e-3) / 1e12
    # DRAM traffic / algorithmic bytes of the FP64 phases, measured by ncu on
    # the n = 16384 instance of this workload family
    traffic_ratio64 = {"phase1": 1.24, "phase2": 1.11}
    bytes64 = {"phase1": 8.0 * sn + 8.0 * n * k, "phase2": 8.0 * (leaves_el + sn) + 16.0 * n * k}
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        res = run_cpu_baseline(args.cpu_n, k)
        if "error" not in res:
            cpu = {"value": res["matmat_gbs"], "unit": "GB/s", "cores": res["threads"],
                   "kind": "reference",
                   "sample": f"hmat_lib multiply_hodlr_dense k={k} on its own build at "
                             f"n={res['n']} (same kernel family; build {res['build_s']:.2f} s)",
                   "build_s": res["build_s"], "cpu": res.get("cpu"),
                   "matvec_n1024_us": res.get("matvec_n1024_us"),
                   "hxh_n4096_s": res.get("hxh_n4096_s")}
        else:
            cpu = {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": "failed: " + res["error"]}
    line = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "s8 slices -> s32 on tensor cores (6 slices, 21 products), f64 result",
        "data": "synthetic", "precision": "mixed",
        "config": {"workload": WORKLOAD if args.n is None else f"matern2d_n{n}", "n": n,
                   "height": h, "leaf": n // (1 << h), "k": k,
                   "tol": tol, "kernel": "matern32 l=0.1 +1e-2 I, 2D Morton points seed 1",
                   "l2": "inputs larger than L2 (factors + X > 126 MB), no flush",
                   "parallelism": f"replicas{world}"},
        "build_s": build_s,
        "build": {"plain": dict(seconds=build_s, rel_err_vs_dense=rel_err,
                                first_build_in_process_s=build_s_first, **plain_stats),
                  "learned": dict(seconds=build_s_learned, rel_err_vs_dense=rel_err_learned,
                                  first_build_in_process_s=build_s_learned_first,
                                  max_rank_diff_vs_plain=int(np.max(np.abs(ranks_l - ranks))),
                                  **learned_stats),
                  "learned_mixed": dict(seconds=build_s_lm, rel_err_vs_dense=rel_err_lm,
                                        max_rank_diff_vs_plain=int(np.max(np.abs(ranks_lm - ranks))),
                                        options="learned_ranks=1, build_precision=1",
                                        **lm_stats),
                  "speedup_learned_mixed_vs_plain": build_s / build_s_lm,
                  "matrix_free": dict(seconds=build_s_mf, max_rank_diff_vs_plain=mf_rank_diff,
                                      input="points only (hodlr_b200_build_kernel_dev)",
                                      **mf_stats),
                  "speedup_learned_vs_plain": build_s / build_s_learned,
                  "model": "hmat_lib_b200/rank_model.f32 (MLP 8-64-64-1, trained by the "
                           "library's GPU kernels)",
                  "roofline_plain": build_roofline(plain_stats, build_s, storage, peak64,
                                                   measured_peaks().get("hbm_gbs", 6650.0)),
                  "roofline_learned": build_roofline(learned_stats, build_s_learned, storage,
                                                     peak64,
                                                     measured_peaks().get("hbm_gbs", 6650.0))},
        "rel_err_vs_dense": rel_err,
        "rel_err_mixed_vs_fp64": rel_err_mixed_vs_fp64,
        "solve": solve_info,
        **side,
        "tree": {"max_rank": info["max_rank"], "storage_doubles": storage,
                 "ranks_by_depth": [int(max(ranks[2 * ((1 << d) - 1):2 * ((1 << (d + 1)) - 1)]))
                                    for d in range(h)]},
        "gflops": flops_step / (ms_step * 1e-3) / 1e9,
        "roofline": {"bound": "tensor", "kernel": f"ozaki_gemm_kernel ({dom})",
                     "achieved": achieved, "peak": peak_i8, "unit": "TOPS (int8)",
                     "frac": achieved / peak_i8,
                     "achieved_incl_slicing": achieved_phase,
                     "frac_incl_slicing": achieved_phase / peak_i8,
                     "traffic": traffic_ratio_i8[dom] * int8_bytes[dom],
                     "traffic_source": "ncu DRAM bytes / operand bytes of this kernel at "
                                       "n = 16384, times the operand bytes at this n",
                     "int8_operand_bytes": int8_bytes[dom],
                     "int8_operand_bytes_by_phase": int8_bytes,
                     "peak_source": peak_src,
                     "phase_ms": {"phase1": rmx["p1"], "phase2": rmx["p2"]},
                     "kernel_ms": {"phase1": rmx["k1"], "phase2": rmx["k2"]}},
        "fp64": {"value": value_fp64, "unit": "GB/s", "ms_per_step": r64["ms"],
                 "gflops": flops_step / (r64["ms"] * 1e-3) / 1e9,
                 "e2e": bytes_step / e2e_s_fp64 / 1e9,
                 "roofline": {"bound": "fp64", "kernel": f"gemm_f64_mma_kernel ({dom64})",
                              "achieved": achieved64, "peak": peak64, "unit": "TFLOP/s",
                              "frac": achieved64 / peak64,
                              "traffic": traffic_ratio64[dom64] * bytes64[dom64],
                              "traffic_source": "ncu DRAM bytes / algorithmic bytes at "
                                                "n = 16384, times the bytes at this n",
                              "algorithmic_bytes": bytes64[dom64],
                              "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                              "phase_ms": {"phase1": r64["p1"], "phase2": r64["p2"]}},
                 "gpu_launches": r64["launches"]},
        "speedup_mixed_vs_fp64": r64["ms"] / rmx["ms"],
        "clocks": rmx["clocks"],
        "e2e": {"value": e2e, "unit": "GB/s", "h2d_bytes_per_step": int(8 * n * k),
                "d2h_bytes_per_step": int(8 * n * k), "ms_per_step": e2e_s * 1e3,
                "path": "multiply_hodlr_dense, option matmat_precision=1"},
        "gpu_launches": rmx["launches"],
        "cpu_baseline": cpu,
        "batch": batch,
        "exp3d_n65536": exp3d,
    }
    print(json.dumps(line))
    host_tree.free()
    tree.free()
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
