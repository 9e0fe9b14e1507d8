"""Matrix-free construction (hodlr_b200_build_kernel_dev): the tree of a
kernel matrix built from its points without forming the matrix matches the
tree built from the same matrix formed densely on the device.  The entries
are computed by the same function, so the two builds differ only where the
sketch products split K and add partial sums with atomics (in an order that
varies from run to run, for two dense builds as well): same ranks (a
singular value within rounding of the threshold may move one), products
equal to rounding."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import rank_model as RM
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, HodlrError
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu

KIND = {"gaussian": 0, "matern32": 1, "exponential": 2}


def _points(n, dim, seed):
    import torch
    pts = W.points_morton(n, dim, seed) if dim > 1 else W.points_1d_sorted(n, seed)
    return pts, torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).cuda()


def _dense(d_pts, n, dim, kind, length, diag):
    import torch
    a = torch.empty(n * n, dtype=torch.float64, device="cuda")
    assert abi.load().hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, dim,
                                                   KIND[kind], length, diag,
                                                   C.c_void_p(a.data_ptr()), n, None) == 0
    torch.cuda.synchronize()
    return a


def _product(dt, x):
    import torch
    n, k = x.shape
    xd = torch.from_numpy(np.asfortranarray(x)).cuda().t().contiguous().t()
    y = torch.zeros_like(xd)
    dt.matmat(xd.data_ptr(), k, n, y.data_ptr(), n)
    torch.cuda.synchronize()
    return y.cpu().numpy()


CASES = [("gaussian", 1, 1024, 3, 0.2, 1.0, 1e-10),      # the smallest workload
         ("matern32", 2, 4096, 5, 0.1, 1e-2, 1e-8),      # sketched blocks
         ("exponential", 3, 2048, 4, 0.15, 1e-2, 1e-8)]


@pytest.mark.parametrize("kind,dim,n,h,length,diag,tol", CASES, ids=[c[0] for c in CASES])
def test_matrix_free_equals_dense_build(kind, dim, n, h, length, diag, tol):
    pts, d_pts = _points(n, dim, 7)
    a = _dense(d_pts, n, dim, kind, length, diag)
    td = DeviceTree.build(a.data_ptr(), n, n, h, tol)
    tf = DeviceTree.build_kernel(d_pts.data_ptr(), n, dim, KIND[kind], length, diag, h, tol)
    assert np.max(np.abs(td.ranks() - tf.ranks())) <= 1
    x = np.random.default_rng(3).standard_normal((n, 12))
    yd, yf = _product(td, x), _product(tf, x)
    assert O.rel_fro(yf, yd) < 1e-12
    # and both approximate the dense product
    ad = a.view(n, n).cpu().numpy().T
    assert O.rel_fro(yf, ad @ x) < 50 * tol
    td.free()
    tf.free()


def test_matrix_free_learned_build():
    """The rank model's features are sketched from the generated matrix too."""
    lib = abi.load()
    n, h, length = 4096, 5, 0.1
    pts, d_pts = _points(n, 2, 9)
    RM.load_default()
    lib.hodlr_b200_set_option(b"learned_ranks", 1.0)
    lib.hodlr_b200_set_option(b"kernel_length", length)
    try:
        a = _dense(d_pts, n, 2, "matern32", length, 1e-2)
        td = DeviceTree.build(a.data_ptr(), n, n, h, 1e-8)
        tf = DeviceTree.build_kernel(d_pts.data_ptr(), n, 2, 1, length, 1e-2, h, 1e-8)
    finally:
        lib.hodlr_b200_set_option(b"learned_ranks", 0.0)
        lib.hodlr_b200_set_option(b"kernel_length", 0.0)
        RM.set_model(None)
    assert np.max(np.abs(td.ranks() - tf.ranks())) <= 1
    x = np.random.default_rng(4).standard_normal((n, 4))
    assert O.rel_fro(_product(tf, x), _product(td, x)) < 1e-12
    td.free()
    tf.free()


def test_matrix_free_argument_errors():
    lib = abi.load()
    out = C.c_void_p()
    ierr = C.c_int(0)
    _, d_pts = _points(256, 2, 1)
    for args in [(2, 256, None, None, 2, 1, 0.1),            # no points
                 (2, 256, None, d_pts.data_ptr(), 2, 3, 0.1),  # unknown kernel
                 (2, 256, None, d_pts.data_ptr(), 2, 1, 0.0),  # zero length
                 (2, 256, None, d_pts.data_ptr(), 0, 1, 0.1)]:  # no dimension
        h, n, ms, p, dim, kind, length = args
        r = lib.hodlr_b200_build_kernel_dev(h, n, ms, C.c_void_p(p), dim, kind, length, 1e-2,
                                            1e-8, 0, None, C.byref(out), C.byref(ierr))
        assert r == abi.INPUT_ERROR and ierr.value == abi.INPUT_ERROR
    with pytest.raises(HodlrError) as e:     # leaf sizes that do not add up
        DeviceTree.build_kernel(d_pts.data_ptr(), 256, 2, 1, 0.1, 1e-2, 1, 1e-8, ms=[100, 100])
    assert e.value.code == abi.INPUT_ERROR


def test_kernel_block_matches_full_matrix():
    """hodlr_b200_kernel_block_dev gives exactly the block of the full kernel
    matrix at its origin (padded leading dimension, diagonal crossing the
    block), and rejects blocks that leave the matrix."""
    import ctypes as C

    import torch

    from hmat_lib_b200 import abi
    lib = abi.load()
    n = 700
    pts = W.points_morton(n, 3, seed=9)
    d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).cuda()
    full = torch.empty(n * n, dtype=torch.float64, device="cuda")
    assert lib.hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, 3, 2, 0.15, 1e-2,
                                            C.c_void_p(full.data_ptr()), n, None) == 0
    r0, c0, rows, cols, ld = 100, 90, 250, 333, 260
    blk = torch.full((cols, ld), float("nan"), dtype=torch.float64, device="cuda")
    assert lib.hodlr_b200_kernel_block_dev(C.c_void_p(d_pts.data_ptr()), n, 3, 2, 0.15, 1e-2,
                                           r0, c0, rows, cols, C.c_void_p(blk.data_ptr()), ld,
                                           None) == 0
    torch.cuda.synchronize()
    a = full.view(n, n).cpu().numpy().T                    # column-major -> numpy
    b = blk.cpu().numpy().T[:rows]
    assert np.array_equal(b, a[r0:r0 + rows, c0:c0 + cols])
    assert lib.hodlr_b200_kernel_block_dev(C.c_void_p(d_pts.data_ptr()), n, 3, 2, 0.15, 1e-2,
                                           n - 10, 0, 11, 5, C.c_void_p(blk.data_ptr()), ld,
                                           None) == abi.INPUT_ERROR
