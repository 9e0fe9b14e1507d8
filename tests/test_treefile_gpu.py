"""On-disk trees (hodlr_b200_tree_save / hodlr_b200_tree_load): a saved and
reloaded tree has the same geometry, ranks and factors, and gives bit-equal
products; truncated, corrupted or foreign files are rejected with
INPUT_ERROR."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, HodlrError, Tree
from hmat_lib_b200.tree import TreeData
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu


def _built(n=2048, h=4):
    import torch
    pts = W.points_morton(n, 2, seed=5)
    a = torch.from_numpy(np.asfortranarray(W.kernel_matrix(pts, "matern32", 0.1, 1e-2))).cuda()
    torch.cuda.synchronize()
    return DeviceTree.build(a.data_ptr(), n, n, h, 1e-8)


def _product(dt, x):
    import torch
    n, k = x.shape
    xd = torch.from_numpy(np.asfortranarray(x)).cuda().t().contiguous().t()
    y = torch.zeros_like(xd)
    dt.matmat(xd.data_ptr(), k, n, y.data_ptr(), n)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def test_round_trip_of_a_built_tree(tmp_path):
    dt = _built()
    path = tmp_path / "tree.hodlr"
    dt.save(path)
    back = DeviceTree.load(path)
    assert back.info() == dt.info()
    assert np.array_equal(back.ranks(), dt.ranks())
    x = np.random.default_rng(1).standard_normal((2048, 24))
    assert np.array_equal(_product(back, x), _product(dt, x))
    a, b = dt.to_host(), back.to_host()
    da, db = a.data(), b.data()
    assert all(np.array_equal(p, q) for p, q in zip(da.leaves, db.leaves))
    for key in da.blocks:
        for p, q in zip(da.blocks[key], db.blocks[key]):
            assert np.array_equal(p, q)
    a.free(); b.free(); back.free(); dt.free()


def test_round_trip_of_uneven_leaves_and_zero_ranks(tmp_path):
    """Leaf sizes given per leaf, some blocks of rank 0."""
    rng = np.random.default_rng(2)
    sizes = [40, 24, 64, 8]
    td = TreeData(2, sizes, [rng.standard_normal((s, s)) for s in sizes])
    for d in range(2):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            for c in (1, 2):
                m, nn = (top, size - top) if c == 1 else (size - top, top)
                r = 0 if (d + j + c) % 3 == 0 else int(rng.integers(1, 6))
                td.blocks[(d, j, c)] = (rng.standard_normal((m, r)), rng.standard_normal((nn, r)))
    t = Tree.from_tree_data(td)
    dt = DeviceTree.of_host(t)
    path = tmp_path / "uneven.hodlr"
    dt.save(path)
    back = DeviceTree.load(path)
    x = rng.standard_normal((136, 5))
    got = _product(back, x)
    assert np.array_equal(got, _product(dt, x))
    assert O.rel_fro(got, O.multiply_dense(td, x)) < 1e-13
    back.free(); dt.free(); t.free()


def test_damaged_files_are_rejected(tmp_path):
    dt = _built(1024, 3)
    path = tmp_path / "tree.hodlr"
    dt.save(path)
    raw = path.read_bytes()
    cases = {
        "truncated": raw[:-100],
        "flipped": raw[:len(raw) // 2] + bytes([raw[len(raw) // 2] ^ 1]) + raw[len(raw) // 2 + 1:],
        "foreign": b"not a tree at all" * 10,
        "empty": b"",
    }
    for name, blob in cases.items():
        bad = tmp_path / f"{name}.hodlr"
        bad.write_bytes(blob)
        with pytest.raises(HodlrError) as e:
            DeviceTree.load(bad)
        assert e.value.code == abi.INPUT_ERROR, name
    with pytest.raises(HodlrError):
        DeviceTree.load(tmp_path / "missing.hodlr")
    dt.free()
