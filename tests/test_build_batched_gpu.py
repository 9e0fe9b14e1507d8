"""Batched construction (hodlr_b200_build_batched_dev): many trees of uneven
size built in shared launches come out as each tree's own build
(hodlr_b200_build_dev) -- same ranks, same products within 1e-12 -- and as
hmat_lib's CPU oracle would build them; an empty batch and invalid inputs
are handled."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, HodlrError
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu


def test_batched_build_equals_single_builds():
    import torch
    items = W.uneven_batch(12, seed=5)
    # smaller trees than the benchmark batch, same families
    for it in items:
        it["n"] = it["n"] // 4
        it["height"] = max(1, (it["n"] // 128).bit_length() - 1)
        it["points"] = it["points"][:it["n"]]
    mats = []
    for it in items:
        a = W.kernel_matrix(np.sort(it["points"][:, 0])[:, None], "exponential", it["length"], 0.0)
        mats.append(torch.from_numpy(np.asfortranarray(a)).cuda())
    torch.cuda.synchronize()
    ns = [it["n"] for it in items]
    hs = [it["height"] for it in items]
    batch = DeviceTree.build_batched([m.data_ptr() for m in mats], ns, ns, hs, 1e-8)
    assert len(batch) == len(items)
    for it, m, tb in zip(items, mats, batch):
        n, h = it["n"], it["height"]
        ts = DeviceTree.build(m.data_ptr(), n, n, h, 1e-8)
        assert np.array_equal(tb.ranks(), ts.ranks())
        x = torch.randn(5, n, dtype=torch.float64, device="cuda")
        yb, ys = torch.zeros_like(x), torch.zeros_like(x)
        tb.matmat(x.data_ptr(), 5, n, yb.data_ptr(), n)
        ts.matmat(x.data_ptr(), 5, n, ys.data_ptr(), n)
        torch.cuda.synchronize()
        assert O.rel_fro(yb.cpu().numpy(), ys.cpu().numpy()) < 1e-12
        dense = m.cpu().numpy()
        want = dense @ x.cpu().numpy().T
        assert O.rel_fro(yb.cpu().numpy().T, want) < 1e-7
        ts.free()
        tb.free()


def test_batched_build_edge_cases(lib):
    out = (C.c_void_p * 1)()
    ierr = C.c_int(-1)
    assert lib.hodlr_b200_build_batched_dev(0, None, None, None, None, 1e-8, None, out,
                                            C.byref(ierr)) == abi.SUCCESS
    assert ierr.value == abi.SUCCESS
    import torch
    a = torch.eye(256, dtype=torch.float64, device="cuda")
    with pytest.raises(HodlrError) as e:
        DeviceTree.build_batched([a.data_ptr()], [256], [100], [1], 1e-8)   # ld < n
    assert e.value.code == abi.INPUT_ERROR
