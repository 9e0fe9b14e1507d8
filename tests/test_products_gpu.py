"""Device parity of the HODLR products through the C-ABI (multiply_vector,
multiply_hodlr_dense, multiply_hodlr_transpose_dense, multiply_dense_hodlr
and the subtree variants) against the CPU oracle and the reference's
known answers.  FP64 throughout; tolerance: 1e-10 absolute for hmat_lib's
known answers (its DELTA), 1e-12 relative Frobenius against the oracle."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, Tree
from hmat_lib_b200.tree import TreeData
from oracle import hodlr_oracle as O

import cases as K

pytestmark = pytest.mark.gpu

REL = 1e-12


def random_tree(n, h, seed, ms=None, max_rank=12, zero_rank_every=0):
    """A caller-assembled HODLR with random leaves and factors."""
    rng = np.random.default_rng(seed)
    sizes = list(ms) if ms is not None else O.block_sizes_halves(n, h)
    td = TreeData(h, sizes)
    for s in sizes:
        td.leaves.append(rng.standard_normal((s, s)))
    idx = 0
    for d in range(h):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            for c in (1, 2):
                m, nn = (top, size - top) if c == 1 else (size - top, top)
                r = int(rng.integers(1, max_rank + 1))
                r = min(r, max(min(m, nn), 1))
                if zero_rank_every and idx % zero_rank_every == 0:
                    r = 0
                td.blocks[(d, j, c)] = (rng.standard_normal((m, r)), rng.standard_normal((nn, r)))
                idx += 1
    return td


@pytest.mark.parametrize("n,h,k", [(21, 1, 1), (21, 3, 5), (100, 2, 17), (257, 4, 64),
                                   (1000, 3, 129), (2048, 4, 256)])
def test_products_match_oracle(n, h, k):
    td = random_tree(n, h, seed=n + k)
    t = Tree.from_tree_data(td)
    x = np.asfortranarray(np.random.default_rng(1).standard_normal((n, k)))
    assert O.rel_fro(t.matmat(x, "N"), O.multiply_dense(td, x)) < REL
    assert O.rel_fro(t.matmat(x, "T"), O.multiply_transpose_dense(td, x)) < REL
    xl = np.asfortranarray(x.T)
    assert O.rel_fro(t.matmat(xl, "L"), O.multiply_dense_hodlr(td, xl)) < REL
    assert O.rel_fro(t.matvec(x[:, 0].copy()), O.multiply_dense(td, x[:, 0])) < REL
    t.free()


def test_products_custom_sizes_and_zero_ranks():
    ms = [3, 1, 7, 2, 9, 4, 1, 5]
    n = sum(ms)
    td = random_tree(n, 3, seed=5, ms=ms, zero_rank_every=3)
    t = Tree.from_tree_data(td)
    x = np.asfortranarray(np.random.default_rng(2).standard_normal((n, 6)))
    assert O.rel_fro(t.matmat(x, "N"), O.multiply_dense(td, x)) < REL
    assert O.rel_fro(t.matmat(x, "T"), O.multiply_transpose_dense(td, x)) < REL
    xl = np.asfortranarray(x.T)
    assert O.rel_fro(t.matmat(xl, "L"), O.multiply_dense_hodlr(td, xl)) < REL


def test_leading_dimensions_and_out_null(lib):
    """ld > rows on input and output; out == NULL returns a malloc'd result
    (hmat_lib src/dense_algebra.c:374-380)."""
    n, h, k, ldx, ldy = 300, 3, 9, 311, 305
    td = random_tree(n, h, seed=9)
    t = Tree.from_tree_data(td)
    x = np.asfortranarray(np.random.default_rng(3).standard_normal((ldx, k)))
    y = np.zeros((ldy, k), order="F")
    ierr = C.c_int(-1)
    p = lib.multiply_hodlr_dense(t.tp, x.ctypes.data_as(abi.DP), k, ldx,
                                 y.ctypes.data_as(abi.DP), ldy, C.byref(ierr))
    assert ierr.value == abi.SUCCESS and p
    want = O.multiply_dense(td, np.ascontiguousarray(x[:n]))
    assert O.rel_fro(y[:n], want) < REL
    p2 = lib.multiply_hodlr_dense(t.tp, x.ctypes.data_as(abi.DP), k, ldx, None, n, C.byref(ierr))
    assert ierr.value == abi.SUCCESS
    got = np.ctypeslib.as_array(p2, shape=(n * k,)).reshape((k, n)).T.copy()
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    libc.free(C.cast(p2, C.c_void_p))
    assert O.rel_fro(got, want) < REL


def test_input_errors(lib):
    td = random_tree(30, 2, seed=1)
    t = Tree.from_tree_data(td)
    x = np.zeros(30)
    ierr = C.c_int(-1)
    assert not lib.multiply_vector(None, abi.as_dp(x), None, C.byref(ierr))
    assert ierr.value == abi.INPUT_ERROR
    ierr.value = -1
    assert not lib.multiply_vector(t.tp, abi.as_dp(x), abi.as_dp(x), C.byref(ierr))
    assert ierr.value == abi.INPUT_ERROR
    ierr.value = -1
    assert not lib.multiply_hodlr_dense(t.tp, None, 1, 30, None, 30, C.byref(ierr))
    assert ierr.value == abi.INPUT_ERROR


def test_subtree_products(lib):
    """multiply_internal_node_dense / _transpose_dense /
    multiply_dense_internal_node on the root and on an inner node
    (hmat_lib src/dense_algebra.c:492, 710, 1087)."""
    n, h, k = 400, 4, 7
    td = random_tree(n, h, seed=4)
    t = Tree.from_tree_data(td)
    from hmat_lib_b200.tree import node_at
    for (d, j) in [(0, 0), (1, 1), (2, 2)]:
        sub = O.subtree(td, d, j)
        node = node_at(t.tp, d, j)
        m = sub.n
        x = np.asfortranarray(np.random.default_rng(d).standard_normal((m, k)))
        out = np.zeros((m, k), order="F")
        lib.multiply_internal_node_dense(node, h - d, x.ctypes.data_as(abi.DP), k, m, None, None,
                                         out.ctypes.data_as(abi.DP), m)
        assert O.rel_fro(out, O.multiply_dense(sub, x)) < REL
        lib.multiply_internal_node_transpose_dense(node, h - d, x.ctypes.data_as(abi.DP), k, m,
                                                   None, None, out.ctypes.data_as(abi.DP), m)
        assert O.rel_fro(out, O.multiply_transpose_dense(sub, x)) < REL
        xl = np.asfortranarray(x.T)
        outl = np.zeros((k, m), order="F")
        lib.multiply_dense_internal_node(node, h - d, xl.ctypes.data_as(abi.DP), k, k, None,
                                         None, outl.ctypes.data_as(abi.DP), k)
        assert O.rel_fro(outl, O.multiply_dense_hodlr(sub, xl)) < REL


@pytest.mark.parametrize("height", [1, 2, 3])
def test_known_answer_products(height):
    """hmat_lib tests/unit_tests/test_hodlr_dense_algebra.c:307-560 and
    test_vector_algebra.c:184-215, with the trees built on the GPU."""
    for transpose in (False, True):
        for name, a, x, e in K.laplacian_product_cases(transpose):
            t = Tree.from_dense(a, height, 0.1)
            y = t.matmat(x, "T" if transpose else "N")
            assert np.abs(y - e).max() <= K.DELTA, (name, transpose)
            if not transpose:
                assert np.abs(t.matvec(x[:, 0].copy()) - e[:, 0]).max() <= K.DELTA
                # X H with X = e^T: (H^T e)^T
                yl = t.matmat(np.asfortranarray(x.T), "L")
                assert np.abs(yl - (a.T @ x).T).max() <= 1e-9, name
            t.free()


def test_repeated_products_reuse_device_copy(lib):
    """A tree keeps its device copy between calls; editing a factor in place
    and calling hodlr_b200_sync_tree makes the next product see the edit."""
    td = random_tree(200, 3, seed=12)
    t = Tree.from_tree_data(td)
    x = np.asfortranarray(np.random.default_rng(0).standard_normal((200, 4)))
    y1 = t.matmat(x)
    n0 = lib.hodlr_b200_kernel_launches()
    y2 = t.matmat(x)
    assert lib.hodlr_b200_kernel_launches() > n0
    np.testing.assert_array_equal(y1, y2)
    u, v = td.blocks[(0, 0, 1)]
    t.keep.buffers[0][:] += 0.0    # leaves untouched
    # edit the root's top-right U in place (its buffer is shared with the tree)
    from hmat_lib_b200.tree import node_at
    od = node_at(t.tp, 0, 0).contents.children[1].leaf.contents.data.off_diagonal
    buf = np.ctypeslib.as_array(od.u, shape=(od.m * od.s,))
    buf[1] += 1.0
    assert lib.hodlr_b200_sync_tree(t.tp) == abi.SUCCESS
    td2 = t.data()
    assert O.rel_fro(t.matmat(x), O.multiply_dense(td2, x)) < REL


def test_large_product_against_dense():
    """Size-independent check at a larger size: H X against the dense
    product of the reconstructed matrix (CPU FP64)."""
    n, h, k = 8192, 6, 32
    td = random_tree(n, h, seed=21, max_rank=40)
    t = Tree.from_tree_data(td)
    x = np.asfortranarray(np.random.default_rng(5).standard_normal((n, k)))
    dense = td.to_dense()
    assert O.rel_fro(t.matmat(x, "N"), dense @ x) < 1e-12
    assert O.rel_fro(t.matmat(x, "T"), dense.T @ x) < 1e-12


@pytest.mark.parametrize("chunks", [0, 1, 3, 7])
def test_host_products_in_column_chunks(lib, chunks):
    """multiply_hodlr_dense / multiply_hodlr_transpose_dense with host
    buffers run in column chunks whose copies overlap the products (option
    host_chunks: 0 automatic, 1 one piece, more: that many chunks); every
    chunking gives the oracle's result and leaves the rows past n of the
    output untouched."""
    n, h, k, ldx, ldy = 1000, 3, 200, 1013, 1007
    td = random_tree(n, h, seed=11)
    t = Tree.from_tree_data(td)
    x = np.asfortranarray(np.random.default_rng(12).standard_normal((ldx, k)))
    ierr = C.c_int(-1)
    lib.hodlr_b200_set_option(b"host_chunks", float(chunks))
    try:
        for fn, ref in [(lib.multiply_hodlr_dense, O.multiply_dense),
                        (lib.multiply_hodlr_transpose_dense, O.multiply_transpose_dense)]:
            y = np.full((ldy, k), np.nan, order="F")
            assert fn(t.tp, x.ctypes.data_as(abi.DP), k, ldx, y.ctypes.data_as(abi.DP), ldy,
                      C.byref(ierr))
            assert ierr.value == abi.SUCCESS
            assert O.rel_fro(y[:n], ref(td, np.ascontiguousarray(x[:n]))) < REL
            assert np.isnan(y[n:]).all()
    finally:
        lib.hodlr_b200_set_option(b"host_chunks", 0.0)
    t.free()


def test_host_mixed_product_in_column_chunks(lib):
    """The mixed-precision host product (option matmat_precision = 1) in
    automatic column chunks agrees with the FP64 one to 1e-11."""
    n, h, k = 1024, 3, 256
    td = random_tree(n, h, seed=13)
    t = Tree.from_tree_data(td)
    x = np.asfortranarray(np.random.default_rng(14).standard_normal((n, k)))
    y64 = t.matmat(x, "N")
    lib.hodlr_b200_set_option(b"matmat_precision", 1.0)
    try:
        ymx = t.matmat(x, "N")
    finally:
        lib.hodlr_b200_set_option(b"matmat_precision", 0.0)
    assert O.rel_fro(ymx, y64) < 1e-11
    assert O.rel_fro(y64, O.multiply_dense(td, x)) < REL
    t.free()


@pytest.mark.parametrize("use_kernels", [1, 0])
def test_single_vector_products(lib, use_kernels):
    """One right-hand side (multiply_vector and H X with k = 1) goes through
    the dedicated projection and row kernels (option matvec_kernels = 1, the
    default) or the GEMM engine (0); both match the oracle on uneven leaves
    with zero-rank blocks and on a depth-5 tree."""
    lib.hodlr_b200_set_option(b"matvec_kernels", float(use_kernels))
    try:
        for ms, h, seed in [([3, 1, 7, 2, 9, 4, 1, 5], 3, 21), (None, 5, 22)]:
            n = sum(ms) if ms else 2000
            td = random_tree(n, h, seed=seed, ms=ms, zero_rank_every=3)
            t = Tree.from_tree_data(td)
            x = np.random.default_rng(seed).standard_normal(n)
            want = O.multiply_dense(td, x[:, None])[:, 0]
            assert O.rel_fro(t.matvec(x.copy()), want) < REL
            assert O.rel_fro(t.matmat(np.asfortranarray(x[:, None]), "N")[:, 0], want) < REL
            t.free()
    finally:
        lib.hodlr_b200_set_option(b"matvec_kernels", 1.0)


@pytest.mark.parametrize("k", [1, 24])
def test_repeated_products_replay_graphs(lib, k):
    """On a non-default stream, a product that repeats an earlier call (same
    tree, op, sizes, buffers) is captured once as a CUDA graph and replayed:
    new input values give the same results as direct launches (option
    product_graphs = 0), and the library's launch counter still counts the
    replayed kernels."""
    import torch
    n, h = 2048, 4
    pts = W.points_morton(n, 2, seed=6)
    a = W.kernel_matrix(pts, "matern32", 0.1, 1e-2)
    t = Tree.from_dense(a, h, 1e-8)
    dt = DeviceTree.of_host(t)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    x = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    rng = np.random.default_rng(k)
    results = []
    for it in range(5):
        xv = rng.standard_normal((n, k))
        x.copy_(torch.from_numpy(np.ascontiguousarray(xv.T)))
        torch.cuda.synchronize()
        l0 = lib.hodlr_b200_kernel_launches()
        dt.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh)
        stream.synchronize()
        assert lib.hodlr_b200_kernel_launches() > l0
        results.append((xv, y.cpu().numpy().T.copy()))
    lib.hodlr_b200_set_option(b"product_graphs", 0.0)
    try:
        for xv, got in results:
            x.copy_(torch.from_numpy(np.ascontiguousarray(xv.T)))
            torch.cuda.synchronize()
            dt.matmat(x.data_ptr(), k, n, y.data_ptr(), n, stream=sh)
            stream.synchronize()
            assert O.rel_fro(y.cpu().numpy().T, got) < 1e-14   # split-K atomics: rounding order
    finally:
        lib.hodlr_b200_set_option(b"product_graphs", 1.0)
    dt.free()
    t.free()
