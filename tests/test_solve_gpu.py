"""Direct solver (hodlr_b200_factorize_dev / hodlr_b200_solve_dev) against
numpy's dense solve of the same HODLR matrix (reconstructed from its
factors), on random trees with uneven leaves and zero ranks and on a built
kernel-matrix tree; singular leaves are reported."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, HodlrError, Tree
from hmat_lib_b200.tree import TreeData
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu


def _random_tree(sizes, h, rng, rank_max=8, zero_every=0, scale=1.0):
    n = sum(sizes)
    td = TreeData(h, list(sizes), [rng.standard_normal((s, s)) + 3.0 * np.sqrt(n) * np.eye(s)
                                   for s in sizes])
    cnt = 0
    for d in range(h):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            for c in (1, 2):
                m, nn = (top, size - top) if c == 1 else (size - top, top)
                cnt += 1
                r = 0 if zero_every and cnt % zero_every == 0 else \
                    int(rng.integers(1, min(rank_max, m, nn) + 1))
                td.blocks[(d, j, c)] = (scale * rng.standard_normal((m, r)),
                                        rng.standard_normal((nn, r)))
    return td


def _solve(dt, b):
    import torch
    n, k = b.shape
    bd = torch.from_numpy(np.asfortranarray(b)).cuda().t().contiguous().t()
    x = torch.full_like(bd, float("nan"))
    f = dt.factorize()
    f.solve(bd.data_ptr(), k, n, x.data_ptr(), n)
    torch.cuda.synchronize()
    f.free()
    return x.cpu().numpy()


@pytest.mark.parametrize("sizes,h,zero_every", [
    ([32, 32, 32, 32], 2, 0),
    ([40, 24, 64, 8], 2, 3),
    ([16] * 16, 4, 5),
    ([128] * 8, 3, 0)])
def test_solve_matches_dense_solve(sizes, h, zero_every):
    rng = np.random.default_rng(len(sizes) + h)
    td = _random_tree(sizes, h, rng, zero_every=zero_every)
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    b = rng.standard_normal((sum(sizes), 7))
    x = _solve(dt, b)
    want = np.linalg.solve(td.to_dense(), b)
    assert O.rel_fro(x, want) < 1e-11
    dt.free()
    t.free()


def test_solve_built_kernel_tree():
    """2D Matern kernel + 1e-2 I (n = 4096): residual through the library's
    own product, and agreement with the dense solve of the HODLR."""
    import torch
    n, h = 4096, 5
    pts = W.points_morton(n, 2, seed=11)
    d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).cuda()
    dt = DeviceTree.build_kernel(d_pts.data_ptr(), n, 2, 1, 0.1, 1e-2, h, 1e-8)
    b = np.random.default_rng(5).standard_normal((n, 16))
    x = _solve(dt, b)
    xd = torch.from_numpy(np.asfortranarray(x)).cuda().t().contiguous().t()
    y = torch.zeros_like(xd)
    dt.matmat(xd.data_ptr(), 16, n, y.data_ptr(), n)
    torch.cuda.synchronize()
    assert O.rel_fro(y.cpu().numpy(), b) < 1e-9
    host = dt.to_host()
    want = np.linalg.solve(host.data().to_dense(), b)
    assert O.rel_fro(x, want) < 1e-8
    host.free()
    dt.free()


def test_singular_leaf_is_reported():
    rng = np.random.default_rng(3)
    td = _random_tree([32, 32], 1, rng)
    td.leaves[1] = np.zeros((32, 32))
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    with pytest.raises(HodlrError) as e:
        dt.factorize()
    assert e.value.code == abi.INPUT_ERROR
    assert b"singular" in abi.load().hodlr_b200_last_error()
    dt.free()
    t.free()


def test_solve_argument_errors():
    import torch
    rng = np.random.default_rng(4)
    td = _random_tree([32, 32], 1, rng)
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    f = dt.factorize()
    x = torch.zeros(64, dtype=torch.float64, device="cuda")
    lib = abi.load()
    assert lib.hodlr_b200_solve_dev(f.h, C.c_void_p(x.data_ptr()), 1, 64,
                                    C.c_void_p(x.data_ptr()), 64, None) == abi.INPUT_ERROR
    y = torch.zeros(64, dtype=torch.float64, device="cuda")
    assert lib.hodlr_b200_solve_dev(f.h, C.c_void_p(x.data_ptr()), 1, 10,
                                    C.c_void_p(y.data_ptr()), 64, None) == abi.INPUT_ERROR
    f.free()
    dt.free()
    t.free()


def test_cached_plans_for_several_shapes():
    """Solves with different k and leading dimensions, repeated (the second
    call of each shape reuses its cached plans and scratch)."""
    import torch
    rng = np.random.default_rng(6)
    sizes = [48, 16, 32, 32, 64, 8, 40, 16]
    td = _random_tree(sizes, 3, rng, zero_every=4)
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    f = dt.factorize()
    n = sum(sizes)
    a = td.to_dense()
    for k, ldb, ldx in [(3, n, n), (9, n + 5, n + 2), (3, n, n), (1, n + 1, n), (9, n + 5, n + 2)]:
        b = rng.standard_normal((ldb, k))
        bd = torch.from_numpy(np.asfortranarray(b)).cuda().t().contiguous().t()
        xd = torch.full((ldx, k), float("nan"), dtype=torch.float64).cuda().t().contiguous().t()
        f.solve(bd.data_ptr(), k, ldb, xd.data_ptr(), ldx)
        torch.cuda.synchronize()
        x = xd.cpu().numpy()
        assert O.rel_fro(x[:n], np.linalg.solve(a, b[:n])) < 1e-11
        assert np.isnan(x[n:]).all()          # rows past n untouched
    f.free()
    dt.free()
    t.free()
