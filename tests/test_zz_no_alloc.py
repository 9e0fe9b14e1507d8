"""hodlr_b200_matvec_noalloc_dev: y = H x without allocating anything, for
callers that cannot allocate device memory while they run (a solver whose
memory pool already holds nearly all of HBM, latency-critical code that
cannot take cudaMalloc's implicit device synchronisation).  Its scratch is a
fixed array of device memory inside the library.

Checked through the C-ABI against the existing device product
(hodlr_b200_matmat_dev with one right-hand side) on two calls in a row, on
a height-1 tree and on a tree whose blocks all have rank zero, and for the
clear rejection of trees beyond the array's capacity (too many ranks, too
many blocks) before anything is launched.  Self-contained
so it passes alone in a fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, Tree
from hmat_lib_b200.tree import TreeData
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu

REL = 1e-12   # FP64 relative Frobenius tolerance used by the product tests


def _noalloc(lib, dt, x, y, stream):
    return lib.hodlr_b200_matvec_noalloc_dev(dt.h, C.c_void_p(x.data_ptr()),
                                             C.c_void_p(y.data_ptr()), C.c_void_p(stream))


def test_noalloc_matvec_matches_existing_entry_point():
    import torch

    lib = abi.load()
    n, h = 3000, 4
    pts = W.points_morton(n, 2, seed=5)
    a = W.kernel_matrix(pts, "matern32", 0.2, 1e-2)
    tree = Tree.from_dense(a, h, 1e-8)
    dt = DeviceTree.of_host(tree)
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y_ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    dt.matmat(x.data_ptr(), 1, n, y_ref.data_ptr(), n, stream=sh)
    outs = []
    for _ in range(2):   # two calls in a row share (and reuse) the fixed scratch
        y = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert _noalloc(lib, dt, x, y, sh) == abi.SUCCESS, lib.hodlr_b200_last_error()
        stream.synchronize()
        outs.append(y.cpu().numpy())
    ref = y_ref.cpu().numpy()
    for out in outs:
        assert np.isfinite(out).all()
        assert O.rel_fro(out, ref) < REL
    # and both agree with the CPU oracle of the same tree
    want = O.multiply_dense(tree.data(), x.cpu().numpy())
    assert O.rel_fro(outs[1], want) < REL
    dt.free()
    tree.free()


def test_noalloc_matvec_rejects_tree_beyond_capacity():
    """Ranks summing past the fixed scratch (65536 entries) are rejected with
    INPUT_ERROR and a message, before any launch."""
    import torch

    lib = abi.load()
    n, h = 32768, 8
    rng = np.random.default_rng(0)
    sizes = O.block_sizes_halves(n, h)
    td = TreeData(h, sizes, [rng.standard_normal((s, s)) for s in sizes])
    for d in range(h):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            # full rank on the two deepest levels: 2 x 32768 entries, plus the rest
            r = top if d >= h - 2 else 1
            for c in (1, 2):
                m, nn = (top, size - top) if c == 1 else (size - top, top)
                td.blocks[(d, j, c)] = (rng.standard_normal((m, r)), rng.standard_normal((nn, r)))
    assert sum(u.shape[1] for u, _ in td.blocks.values()) > 65536
    tree = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(tree)
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert _noalloc(lib, dt, x, y, 0) == abi.INPUT_ERROR
    assert b"65536" in lib.hodlr_b200_last_error()
    assert float(y.abs().max()) == 0.0   # nothing launched
    dt.free()
    tree.free()


def _random_tree(sizes, h, rank_of, seed=0):
    rng = np.random.default_rng(seed)
    td = TreeData(h, sizes, [rng.standard_normal((s, s)) for s in sizes])
    for d in range(h):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            r = rank_of(d, top)
            for c in (1, 2):
                m, nn = (top, size - top) if c == 1 else (size - top, top)
                td.blocks[(d, j, c)] = (rng.standard_normal((m, r)), rng.standard_normal((nn, r)))
    return td


@pytest.mark.parametrize("case", ["one_level", "zero_ranks"])
def test_noalloc_matvec_edge_trees(case):
    """The smallest tree (height 1: two leaves, one rank-0 and one rank-5
    block; hmat_lib's allocate_tree takes no height-0 tree) and a tree whose
    blocks all have rank 0 (no projection is launched): same result as the
    existing device product and as the CPU oracle."""
    import torch

    lib = abi.load()
    if case == "one_level":
        n, h = 200, 1
        td = _random_tree([100, 100], h, lambda d, top: 0, seed=1)
        rng = np.random.default_rng(11)
        td.blocks[(0, 0, 2)] = (rng.standard_normal((100, 5)), rng.standard_normal((100, 5)))
    else:
        n, h = 1000, 3
        td = _random_tree(O.block_sizes_halves(n, h), h, lambda d, top: 0, seed=2)
    tree = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(tree)
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y_ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    dt.matmat(x.data_ptr(), 1, n, y_ref.data_ptr(), n)
    for _ in range(2):
        y = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert _noalloc(lib, dt, x, y, 0) == abi.SUCCESS, lib.hodlr_b200_last_error()
        torch.cuda.synchronize()
        assert O.rel_fro(y.cpu().numpy(), y_ref.cpu().numpy()) < REL
    want = O.multiply_dense(td, x.cpu().numpy())
    assert O.rel_fro(y.cpu().numpy(), want) < REL
    dt.free()
    tree.free()


def test_noalloc_matvec_rejects_too_many_blocks():
    """Height 12 has 8190 off-diagonal blocks, past the 4096 offsets the fixed
    scratch holds: INPUT_ERROR and a message before any launch (ranks tiny,
    so only the block count is over)."""
    import torch

    lib = abi.load()
    h = 12
    n = 2 << h                      # leaves of 2 rows
    td = _random_tree(O.block_sizes_halves(n, h), h, lambda d, top: 0, seed=3)
    tree = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(tree)
    x = torch.randn(n, dtype=torch.float64, device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    launches = lib.hodlr_b200_kernel_launches()
    assert _noalloc(lib, dt, x, y, 0) == abi.INPUT_ERROR
    assert lib.hodlr_b200_kernel_launches() == launches
    assert b"4096" in lib.hodlr_b200_last_error()
    assert float(y.abs().max()) == 0.0
    dt.free()
    tree.free()
