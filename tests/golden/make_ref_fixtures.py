"""Generates the full-size reference fixtures of tests/golden/ (run from the
repo root, CPU only): hmat_lib's own FP64 results on two workloads.

    make -C oracle ref64
    python tests/golden/make_ref_fixtures.py --workload matern2d_n32768 [--threads 8]
    python tests/golden/make_ref_fixtures.py --workload exp3d_n8192 [--threads 8]

matern2d_n32768 -> ref_matern2d_n32768.npz: n = 32768 points of [0,1]^2
    (seed 1) in Morton order, Matern-3/2 kernel with length 0.1 plus 1e-2 I,
    depth 8 (leaf 128), tolerance 1e-8.  The unmodified reference cannot
    build this size (its constructor computes scratch sizes and block offsets
    in `int`, hmat_lib src/constructors.c:464, 676), so this runs the copy
    "patched for 64-bit sizes" that oracle/Makefile's `ref64` target builds:
    the same code with only those integers widened.
exp3d_n8192 -> ref_exp3d_n8192.npz: n = 8192 points of [0,1]^3 (seed 4) in
    Morton order, exp(-r / 0.15) plus 1e-2 I, depth 6 (leaf 128), tolerance
    1e-8 -- the family of the n = 65536 learned-rank workload at a size the
    unmodified reference builds.

Stored: the rank of every off-diagonal block (order b = 2(2^d - 1 + j) +
(c - 1), as DeviceTree.ranks() returns them), the reference's
multiply_hodlr_dense of four seeded right-hand sides (X = rhs(n, 4, seed=7),
hmat_lib_b200.workloads.rhs), the relative error of that product against the
dense A X, and how long the reference took.  The kernel matrix is built on
the host in column blocks (same formula as the device generator).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hmat_lib_b200 import abi, workloads as W  # noqa: E402
from hmat_lib_b200.tree import node_at  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "libhmat_ref.so")
REF64 = os.path.join(ROOT, "oracle", "_ref", "libhmat_ref64.so")
FIXTURES = {
    # workload: (n, dim, seed, kind, length, diag, height, library, label)
    "matern2d_n32768": (32768, 2, 1, "matern32", 0.1, 1e-2, 8, REF64,
                        "hmat_lib patched for 64-bit sizes (oracle/Makefile ref64)"),
    "exp3d_n8192": (8192, 3, 4, "exponential", 0.15, 1e-2, 6, REF,
                    "hmat_lib, unmodified (oracle/Makefile)"),
}
X_SEED = 7
X_COLS = 4


def kernel_matrix_blocked(pts: np.ndarray, kind: str, length: float, diag: float,
                          cols: int = 512) -> np.ndarray:
    n = pts.shape[0]
    a = np.empty((n, n), order="F")
    for j0 in range(0, n, cols):
        j1 = min(n, j0 + cols)
        d = pts[:, None, :] - pts[None, j0:j1, :]
        r = np.sqrt(np.einsum("ijk,ijk->ij", d, d))
        a[:, j0:j1] = W.kernel_values(kind, r, length)
    a[np.arange(n), np.arange(n)] += diag
    return a


def block_ranks(tp) -> np.ndarray:
    h = tp.contents.height
    out = np.zeros(2 * ((1 << h) - 1), dtype=np.int32)
    for d in range(h):
        for j in range(1 << d):
            nd = node_at(tp, d, j).contents
            for c in (1, 2):
                out[2 * ((1 << d) - 1 + j) + c - 1] = nd.children[c].leaf.contents.data.off_diagonal.s
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=sorted(FIXTURES), default="matern2d_n32768")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--n", type=int, default=None, help="smaller n (trial runs only)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    n, dim, seed, kind, length, diag, h, libpath, label = FIXTURES[args.workload]
    out_path = args.out or os.path.join(HERE, f"ref_{args.workload}.npz")
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    if not os.path.exists(libpath):
        raise SystemExit(f"{libpath} missing: run make -C oracle (ref64 for the patched copy)")
    lib = abi.load_hmat_abi(libpath)
    libgomp = C.CDLL("libgomp.so.1", mode=C.RTLD_GLOBAL)
    libgomp.omp_set_num_threads(C.c_int(args.threads))
    import sysconfig
    blasdir = os.path.join(sysconfig.get_paths()["purelib"], "opencv_python_headless.libs")
    blas = None
    for name in os.listdir(blasdir):
        if name.startswith("libopenblas"):
            blas = C.CDLL(os.path.join(blasdir, name), mode=C.RTLD_GLOBAL)
    if blas is not None:
        blas.openblas_set_num_threads(C.c_int(1))

    tol = 1e-8
    if args.n is not None:
        n, h = args.n, max(1, (args.n // 128).bit_length() - 1)
    pts = W.points_morton(n, dim, seed)
    t0 = time.perf_counter()
    a = kernel_matrix_blocked(pts, kind, length, diag)
    x = np.asfortranarray(W.rhs(n, X_COLS, seed=X_SEED))
    y_dense = a @ x
    print(f"matrix + dense product: {time.perf_counter() - t0:.1f} s", flush=True)

    ierr = C.c_int(0)
    tp = lib.allocate_tree_monolithic(h, C.byref(ierr))
    assert ierr.value == abi.SUCCESS
    t0 = time.perf_counter()
    # dense_to_tree_hodlr overwrites its input (hmat_lib src/constructors.c:576-580)
    res = lib.dense_to_tree_hodlr(tp, n, None, a.reshape(-1, order="F").ctypes.data_as(abi.DP),
                                  tol, C.byref(ierr))
    build_s = time.perf_counter() - t0
    if ierr.value != abi.SUCCESS or res != 0:
        raise SystemExit(f"dense_to_tree_hodlr: ierr={ierr.value} info={res}")
    print(f"reference build: {build_s:.1f} s", flush=True)
    del a
    ranks = block_ranks(tp)
    if blas is not None:
        blas.openblas_set_num_threads(C.c_int(args.threads))
    y = np.zeros_like(x, order="F")
    t0 = time.perf_counter()
    lib.multiply_hodlr_dense(tp, x.ctypes.data_as(abi.DP), X_COLS, n, y.ctypes.data_as(abi.DP), n,
                             C.byref(ierr))
    matmat_s = time.perf_counter() - t0
    assert ierr.value == abi.SUCCESS
    err = float(np.linalg.norm(y - y_dense) / np.linalg.norm(y_dense))
    cpu = "unknown"
    for line in open("/proc/cpuinfo"):
        if line.startswith("model name"):
            cpu = line.split(":", 1)[1].strip()
            break
    meta = dict(workload=args.workload, n=n, height=h, tol=tol, x_seed=X_SEED, x_cols=X_COLS,
                build_s=build_s, matmat_s_4cols=matmat_s, threads=args.threads, cpu=cpu,
                rel_err_ref_vs_dense=err, library=label)
    np.savez_compressed(out_path, ranks=ranks, y_ref=y, meta=json.dumps(meta))
    print(json.dumps(meta))
    lib.free_tree_hodlr(C.byref(tp))


if __name__ == "__main__":
    main()
