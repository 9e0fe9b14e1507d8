"""Mixed-precision (int8 tensor-core slices, FP64 recombination) HODLR x
dense product against the FP64 device product and the CPU oracle.  The
slicing keeps about 42 bits; the test tolerance is 1e-11 relative Frobenius
against the FP64 product (the FP64 path itself is pinned to the oracle at
1e-12)."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, Tree
from hmat_lib_b200.tree import TreeData
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _products(dt, xn, k):
    import torch
    n = xn.shape[0]
    x = torch.from_numpy(np.ascontiguousarray(xn.T)).cuda()      # column-major n x k
    y64 = torch.zeros_like(x)
    ymx = torch.full_like(x, float("nan"))
    torch.cuda.synchronize()
    dt.matmat(x.data_ptr(), k, n, y64.data_ptr(), n, precision=0)
    dt.matmat(x.data_ptr(), k, n, ymx.data_ptr(), n, precision=1)
    torch.cuda.synchronize()
    assert abi.load().hodlr_b200_check(dt.h, None) == abi.SUCCESS
    return y64.cpu().numpy().T, ymx.cpu().numpy().T


@pytest.mark.parametrize("n,h,k", [(2048, 4, 64), (4096, 5, 17), (4096, 5, 256), (8192, 6, 1)])
def test_mixed_matches_fp64_on_built_tree(n, h, k):
    pts = W.points_morton(n, 2, seed=1)
    a = W.kernel_matrix(pts, "matern32", 0.1, 1e-2)
    t = Tree.from_dense(a, h, 1e-8)
    dt = DeviceTree.of_host(t)
    x = np.random.default_rng(k).standard_normal((n, k))
    y64, ymx = _products(dt, x, k)
    assert np.isfinite(ymx).all()
    assert O.rel_fro(ymx, y64) < TOL
    dt.free()
    t.free()


def test_mixed_tall_leaves_and_random_factors():
    """Leaves of 256 rows (two M tiles per band), random factors of wildly
    different scales per block."""
    rng = np.random.default_rng(7)
    n, h = 2048, 3
    sizes = O.block_sizes_halves(n, h)
    td = TreeData(h, sizes, [rng.standard_normal((s, s)) for s in sizes])
    for d in range(h):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            for c in (1, 2):
                m, nn = (top, size - top) if c == 1 else (size - top, top)
                r = int(rng.integers(1, 90))
                scale = 10.0 ** rng.uniform(-6, 3)
                td.blocks[(d, j, c)] = (scale * rng.standard_normal((m, r)),
                                        rng.standard_normal((nn, r)))
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    x = rng.standard_normal((n, 70))
    y64, ymx = _products(dt, x, 70)
    assert O.rel_fro(ymx, y64) < TOL
    assert O.rel_fro(ymx, O.multiply_dense(td, x)) < TOL
    dt.free()
    t.free()


def test_mixed_rejects_unaligned_leaves(lib):
    td = TreeData(1, [30, 30], [np.eye(30), np.eye(30)])
    td.blocks[(0, 0, 1)] = (np.ones((30, 1)), np.ones((30, 1)))
    td.blocks[(0, 0, 2)] = (np.ones((30, 1)), np.ones((30, 1)))
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    import torch
    x = torch.zeros(60, dtype=torch.float64, device="cuda")
    y = torch.zeros(60, dtype=torch.float64, device="cuda")
    r = lib.hodlr_b200_matmat_dev(dt.h, 0, 1, C.c_void_p(x.data_ptr()), 1, 60,
                                  C.c_void_p(y.data_ptr()), 60, None)
    assert r == abi.INPUT_ERROR
    assert b"multiples of 32" in lib.hodlr_b200_last_error()
    dt.free()
    t.free()


def _products_op(dt, xn, op, ldpad=0):
    """op 1: H^T X (X n x k); op 2: X H (X k x n); leading dimensions padded
    by `ldpad` rows."""
    import torch
    rows, cols = xn.shape
    ld = rows + ldpad
    xfull = np.zeros((cols, ld))
    xfull[:, :rows] = xn.T
    x = torch.from_numpy(xfull).cuda()                 # column-major rows x cols, ld
    y64 = torch.zeros_like(x)
    ymx = torch.full_like(x, float("nan"))
    torch.cuda.synchronize()
    k = cols if op == 1 else rows
    dt.matmat(x.data_ptr(), k, ld, y64.data_ptr(), ld, op=op, precision=0)
    dt.matmat(x.data_ptr(), k, ld, ymx.data_ptr(), ld, op=op, precision=1)
    torch.cuda.synchronize()
    assert abi.load().hodlr_b200_check(dt.h, None) == abi.SUCCESS
    return y64.cpu().numpy().T[:rows], ymx.cpu().numpy().T[:rows]


@pytest.mark.parametrize("op", [1, 2], ids=["HtX", "XH"])
def test_mixed_transpose_and_left_products(op):
    """H^T X and X H on the int8 path (through the cached transposed tree):
    against the FP64 device product within 1e-11 and against the CPU oracle,
    on a nonsymmetric random tree with uneven ranks and scales, with padded
    leading dimensions; the second call reuses the cached transposed tree."""
    rng = np.random.default_rng(11 + op)
    n, h = 2048, 4
    sizes = O.block_sizes_halves(n, h)
    td = TreeData(h, sizes, [rng.standard_normal((s, s)) for s in sizes])
    for d in range(h):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            for c in (1, 2):
                m, nn = (top, size - top) if c == 1 else (size - top, top)
                r = int(rng.integers(0, 70))
                scale = 10.0 ** rng.uniform(-4, 2)
                td.blocks[(d, j, c)] = (scale * rng.standard_normal((m, r)),
                                        rng.standard_normal((nn, r)))
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    k = 37
    x = rng.standard_normal((n, k)) if op == 1 else rng.standard_normal((k, n))
    for ldpad in (0, 3):
        y64, ymx = _products_op(dt, x, op, ldpad)
        assert np.isfinite(ymx).all()
        assert O.rel_fro(ymx, y64) < TOL
    dense = td.to_dense()
    want = dense.T @ x if op == 1 else x @ dense
    assert O.rel_fro(ymx, want) < TOL
    dt.free()
    t.free()


def test_mixed_host_entry_points_all_ops(lib):
    """multiply_hodlr_dense / _transpose_dense / multiply_dense_hodlr with
    option matmat_precision = 1 take the int8 path for every op: same result
    as the FP64 option within 1e-11."""
    n, h = 2048, 4
    pts = W.points_morton(n, 2, seed=2)
    a = W.kernel_matrix(pts, "matern32", 0.1, 1e-2)
    t = Tree.from_dense(a, h, 1e-8)
    rng = np.random.default_rng(3)
    xr = rng.standard_normal((n, 40))
    xl = rng.standard_normal((40, n))
    try:
        out = {}
        for prec in (0, 1):
            lib.hodlr_b200_set_option(b"matmat_precision", float(prec))
            out[prec] = (t.matmat(xr, "N"), t.matmat(xr, "T"), t.matmat(xl, "L"))
    finally:
        lib.hodlr_b200_set_option(b"matmat_precision", 0.0)
    for y64, ymx in zip(out[0], out[1]):
        assert O.rel_fro(ymx, y64) < TOL
    t.free()
