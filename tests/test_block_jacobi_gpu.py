"""The block Jacobi SVD of wide sketch cores (32-column blocks paired
round-robin: Gram matrix of each 64-column pair, its eigenvectors by Jacobi
in shared memory, rotation of the pair's columns), checked through the
build: with option jacobi_block_min_c lowered
so that every sketched core takes the block solver, the tree has the same
ranks (within one, a singular value at the threshold may fall either side)
and the same accuracy against the dense product as with the one-CTA /
cluster solver, and matches hmat_lib's ranks on the 3D exponential
reference fixture."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, lib as hlib
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _build(a, n, h, tol, block_min):
    lib = hlib()
    lib.hodlr_b200_set_option(b"jacobi_block_min_c", float(block_min))
    try:
        return DeviceTree.build(a.data_ptr(), n, n, h, tol)
    finally:
        lib.hodlr_b200_set_option(b"jacobi_block_min_c", 128.0)


@pytest.mark.parametrize("n,h,kind,length", [(4096, 5, "matern32", 0.1),
                                             (8192, 6, "exponential", 0.15)])
def test_block_solver_matches_scalar_solver(n, h, kind, length):
    import torch
    dim = 2 if kind == "matern32" else 3
    pts = W.points_morton(n, dim, seed=4)
    a = torch.from_numpy(np.asfortranarray(W.kernel_matrix(pts, kind, length, 1e-2))).cuda()
    torch.cuda.synchronize()
    t_ref = _build(a, n, h, 1e-8, 1 << 30)      # every core on the scalar solver
    t_blk = _build(a, n, h, 1e-8, 64)           # every sketched core on the block solver
    r_ref, r_blk = t_ref.ranks(), t_blk.ranks()
    assert int(np.abs(r_ref - r_blk).max()) <= 1
    x = np.random.default_rng(0).standard_normal((n, 8))
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    want = a.cpu().numpy() @ x
    errs = []
    for t in (t_ref, t_blk):
        y = torch.zeros_like(xd)
        t.matmat(xd.data_ptr(), 8, n, y.data_ptr(), n)
        torch.cuda.synchronize()
        errs.append(O.rel_fro(y.cpu().numpy().T, want))
    assert errs[1] <= 2.0 * errs[0] + 1e-12, errs
    t_ref.free()
    t_blk.free()


def test_block_solver_against_reference_ranks():
    """The n = 8192 3D exponential workload (hmat_lib's ranks in
    tests/golden/ref_exp3d_n8192.npz), matrix-free, every sketched core on
    the block solver: ranks within one of hmat_lib's, H X within 1e-8 of
    hmat_lib's product."""
    import torch
    ref = np.load(os.path.join(HERE, "golden", "ref_exp3d_n8192.npz"))
    meta = json.loads(str(ref["meta"]))
    n, h = meta["n"], meta["height"]
    lib = hlib()
    pts = W.points_morton(n, 3, 4)
    d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).cuda()
    lib.hodlr_b200_set_option(b"jacobi_block_min_c", 64.0)
    try:
        t = DeviceTree.build_kernel(d_pts.data_ptr(), n, 3, 2, 0.15, 1e-2, h, meta["tol"])
    finally:
        lib.hodlr_b200_set_option(b"jacobi_block_min_c", 128.0)
    assert int(np.abs(t.ranks() - ref["ranks"]).max()) <= 1
    x = W.rhs(n, meta["x_cols"], seed=meta["x_seed"])
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
    y = torch.zeros_like(xd)
    t.matmat(xd.data_ptr(), meta["x_cols"], n, y.data_ptr(), n)
    torch.cuda.synchronize()
    assert O.rel_fro(y.cpu().numpy().T, ref["y_ref"]) < 1e-8
    t.free()
