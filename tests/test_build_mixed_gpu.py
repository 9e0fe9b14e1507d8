"""The build's sketch products (Y = A Omega, B^T = A^T Q) on the int8 tensor
cores (option build_precision = 1): the tree has the ranks of the FP64 build
(within one) and the same accuracy against the dense product, on a 2D
Matern and a 3D exponential matrix, and (uneven leaves, sizes not multiples
of 32) blocks that cannot be sliced fall back to the FP64 GEMMs."""
import numpy as np
import pytest

from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, lib as hlib
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu


def _build(a, n, h, mixed, ms=None):
    lib = hlib()
    lib.hodlr_b200_set_option(b"build_precision", 1.0 if mixed else 0.0)
    try:
        return DeviceTree.build(a.data_ptr(), n, n, h, 1e-8, ms=ms)
    finally:
        lib.hodlr_b200_set_option(b"build_precision", 0.0)


@pytest.mark.parametrize("case", ["matern2d_4096", "exp3d_4096", "uneven_3000"])
def test_int8_sketches_match_fp64_build(case):
    import torch
    ms = None
    if case == "matern2d_4096":
        n, h = 4096, 5
        a = W.kernel_matrix(W.points_morton(n, 2, seed=1), "matern32", 0.1, 1e-2)
    elif case == "exp3d_4096":
        n, h = 4096, 5
        a = W.kernel_matrix(W.points_morton(n, 3, seed=4), "exponential", 0.15, 1e-2)
    else:
        n, h = 3000, 4
        a = W.kernel_matrix(W.points_morton(n, 2, seed=2), "matern32", 0.2, 1e-2)
        ms = [200, 160, 192, 190, 180, 210, 188, 180, 176, 194, 192, 178, 170, 190, 200, 200]
    da = torch.from_numpy(np.asfortranarray(a)).cuda()
    torch.cuda.synchronize()
    t64 = _build(da, n, h, False, ms)
    tmx = _build(da, n, h, True, ms)
    assert int(np.abs(t64.ranks() - tmx.ranks()).max()) <= 1
    x = np.random.default_rng(0).standard_normal((n, 6))
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    want = a @ x
    errs = []
    for t in (t64, tmx):
        y = torch.zeros_like(xd)
        t.matmat(xd.data_ptr(), 6, n, y.data_ptr(), n)
        torch.cuda.synchronize()
        errs.append(O.rel_fro(y.cpu().numpy().T, want))
    assert errs[1] <= 1.5 * errs[0] + 1e-12, errs
    t64.free()
    tmx.free()
