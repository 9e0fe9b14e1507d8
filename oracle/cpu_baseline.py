"""Timed CPU baseline: the unmodified hmat_lib (oracle/_ref/libhmat_ref.so)
on this machine's host cores -- TEST/BENCH INFRASTRUCTURE ONLY.

    python -m oracle.cpu_baseline --n 4096 --height 5 --k 256 --steps 3

Builds a Matern-3/2 kernel matrix on 2D Morton-ordered points (the family of
the n = 32768 benchmark workload, at a size the unmodified reference can
build: its constructor overflows `int` at n = 32768, hmat_lib
src/constructors.c:676; n = 16384 is the largest power of two it builds),
times dense_to_tree_hodlr with OpenMP tasks on every core and one BLAS thread
each, then times multiply_hodlr_dense with a threaded BLAS (the reference's
algebra has no OpenMP).  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--height", type=int, default=None, help="default: leaves of 128")
    ap.add_argument("--k", type=int, default=256)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--no-side", action="store_true",
                    help="skip the n = 1024 H x and n = 4096 H x H timings")
    ap.add_argument("--batch-sample", type=int, default=0,
                    help="time this many instances per size class of the uneven batch")
    args = ap.parse_args()
    if args.height is None:
        args.height = max(1, (args.n // 128).bit_length() - 1)

    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    import numpy as np

    from hmat_lib_b200 import workloads as W
    from oracle import ref_lib

    ref_lib.load()
    ref_lib.set_omp_threads(args.threads)
    ref_lib.set_blas_threads(1)
    w = W.WORKLOADS["matern2d_n32768"]
    pts = W.points_morton(args.n, 2, w["seed"])
    a = W.kernel_matrix_blocked(pts, w["kind"], w["length"], w["diag"])
    t0 = time.perf_counter()
    tree = ref_lib.build(a, args.height, args.tol)
    del a
    build_s = time.perf_counter() - t0
    td = tree.data()
    storage = td.storage()
    x = np.asfortranarray(W.rhs(args.n, args.k, seed=1))
    ref_lib.set_blas_threads(args.threads)
    for _ in range(args.warmup):
        ref_lib.multiply_dense(tree, x, "N")
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref_lib.multiply_dense(tree, x, "N")
        times.append(time.perf_counter() - t0)
    step = float(np.sum(times) / len(times))      # all timed steps, like the GPU arm
    nbytes = 8.0 * storage + 16.0 * args.n * args.k
    flops = 2.0 * args.k * storage
    out = dict(
        n=args.n, height=args.height, k=args.k, tol=args.tol, threads=args.threads,
        build_s=build_s, matmat_s=step, matmat_gbs=nbytes / step / 1e9,
        matmat_gflops=flops / step / 1e9, storage=int(storage),
        max_rank=int(max(td.ranks().values())),
        cpu=_cpu_model())
    if not args.no_side:
        out.update(side_workloads(args.threads))
    if args.batch_sample > 0:
        out["batch_sample"] = batch_sample(args.batch_sample, args.threads)
    print(json.dumps(out))


def batch_sample(per_class: int, threads: int) -> dict:
    """The uneven batch (512 trees, n in {1024, 2048, 4096, 8192}, seed 2),
    sampled: the first `per_class` instances of each size, each built by the
    reference and timed in multiply_hodlr_dense with its own k.  Reports the
    sample's bytes and time per class and the whole batch's step time
    extrapolated class by class (count in the batch x mean time of the
    class's sample)."""
    import numpy as np

    from hmat_lib_b200 import workloads as W
    from oracle import ref_lib

    insts = W.uneven_batch(512, seed=2)
    classes = {}
    for it in insts:
        classes.setdefault(it["n"], []).append(it)
    res = {"per_class": {}, "sample": f"first {per_class} instances of each size class"}
    est_s, est_bytes = 0.0, 0.0
    for n in sorted(classes):
        times, nbytes = [], []
        for it in classes[n][:per_class]:
            a = W.kernel_matrix_blocked(it["points"], "exponential", it["length"], 0.0)
            ref_lib.set_omp_threads(threads)
            ref_lib.set_blas_threads(1)
            t = ref_lib.build(a, it["height"], it["tol"])
            del a
            td = t.data()
            x = np.asfortranarray(np.random.default_rng(0).standard_normal((n, it["k"])))
            ref_lib.set_blas_threads(threads)
            ref_lib.multiply_dense(t, x, "N")
            t0 = time.perf_counter()
            for _ in range(3):
                ref_lib.multiply_dense(t, x, "N")
            times.append((time.perf_counter() - t0) / 3)
            nbytes.append(8.0 * td.storage() + 16.0 * n * it["k"])
            t.free()
        count = len(classes[n])
        res["per_class"][str(n)] = {"count": count, "sampled": len(times),
                                    "mean_s": float(np.mean(times)),
                                    "mean_bytes": float(np.mean(nbytes))}
        est_s += count * float(np.mean(times))
        est_bytes += count * float(np.mean(nbytes))
    res["step_s_extrapolated"] = est_s
    res["gbs_extrapolated"] = est_bytes / est_s / 1e9
    return res


def side_workloads(threads: int) -> dict:
    """The reference on the two smaller workloads of the hot path: H x on the
    n = 1024 Gaussian tree (the workload's own size), and H_A H_B on the
    Gaussian / Matern-3/2 pair on sorted 1D points at n = 4096 (depth 5; the
    n = 16384 pair takes the reference minutes to build)."""
    import numpy as np

    from hmat_lib_b200 import workloads as W
    from oracle import ref_lib

    res = {}
    w = W.WORKLOADS["gauss1d_n1024"]
    pts = W.workload_points("gauss1d_n1024")
    a = W.kernel_matrix(pts, w["kind"], w["length"], w["diag"])
    ref_lib.set_omp_threads(threads)
    ref_lib.set_blas_threads(1)
    t = ref_lib.build(a, w["height"], w["tol"])
    ref_lib.set_blas_threads(threads)
    x = np.random.default_rng(0).standard_normal(w["n"])
    for _ in range(20):
        ref_lib.multiply_vector(t, x)
    reps = 200
    t0 = time.perf_counter()
    for _ in range(reps):
        ref_lib.multiply_vector(t, x)
    res["matvec_n1024_us"] = (time.perf_counter() - t0) / reps * 1e6
    n = 4096
    pts, ka, kb = W.hxh_pair(n, seed=3)
    ref_lib.set_blas_threads(1)
    ta = ref_lib.build(W.kernel_matrix(pts, *ka), 5, 1e-8)
    tb = ref_lib.build(W.kernel_matrix(pts, *kb), 5, 1e-8)
    ref_lib.set_blas_threads(threads)
    t0 = time.perf_counter()
    ref_lib.multiply_hodlr_hodlr(ta, tb, 1e-8)
    res["hxh_n4096_s"] = time.perf_counter() - t0
    return res


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


if __name__ == "__main__":
    main()
