"""Device parity of multiply_hodlr_hodlr (HODLR x HODLR with recompression)
through the C-ABI: hmat_lib's known answers
(tests/unit_tests/test_hodlr_hodlr_algebra.c:59-338: exact products at
n = 21, tol 1e-8, element-wise within its 1e-10 DELTA, ranks equal to the
expected tree's) and the reference library's ranks and products on seeded
kernel matrices (tests/golden/reference_outputs.npz); hmat_lib's
recompression golden values through the device recompression routine."""
import numpy as np
import pytest

from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import Tree
from oracle import hodlr_oracle as O

import cases as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("height", [1, 2, 3])
def test_hxh_known_answers(height):
    for name, a, b, e in K.hxh_cases():
        ta = Tree.from_dense(np.asfortranarray(a), height, 1e-8)
        tb = ta if name == "L x L" else Tree.from_dense(np.asfortranarray(b), height, 1e-8)
        tc = ta.hxh(tb, 1e-8)
        td = tc.data()
        assert np.abs(td.to_dense() - e).max() <= K.DELTA, name
        te = O.dense_to_tree(np.asarray(e), height, 1e-8)
        for key, (u, v) in td.blocks.items():
            want = te.blocks[key][0].shape[1]
            if np.abs(te.blocks[key][0]).max() > 0:
                assert u.shape[1] == want, (name, key)
        tc.free()
        if tb is not ta:
            tb.free()
        ta.free()


HXH_CASES = [
    ("g21_h3", 21, 3, "gaussian", 0.2, 1.0, 1e-10),
    ("g155_h4", 155, 4, "gaussian", 0.2, 1.0, 1e-10),
    ("m300_h3", 300, 3, "matern32", 0.1, 1e-2, 1e-8),
    ("e517_h4", 517, 4, "exponential", 0.3, 0.0, 1e-8),
    ("g1024_h3", 1024, 3, "gaussian", 0.2, 1.0, 1e-10),
]


@pytest.mark.parametrize("case", HXH_CASES, ids=lambda c: c[0])
def test_hxh_matches_reference(case):
    name, n, h, kind, length, diag, tol = case
    ref = K.reference_outputs()
    pts = W.points_1d_sorted(n, seed=7)
    a = W.kernel_matrix(pts, kind, length, diag)
    b = W.kernel_matrix(pts, "matern32", 0.2, 1.0)
    ta, tb = Tree.from_dense(a, h, tol), Tree.from_dense(b, h, tol)
    tc = ta.hxh(tb, 1e-8)
    td = tc.data()
    ranks = np.array([td.blocks[k][0].shape[1] for k in sorted(td.blocks)])
    np.testing.assert_array_equal(ranks, ref[f"{name}/hxh_ranks"])
    x = W.rhs(n, 3, seed=11)
    assert O.rel_fro(O.multiply_dense(td, x), ref[f"{name}/hxh_y"]) < 1e-10
    # the product tree also multiplies on the device like any other tree
    assert O.rel_fro(tc.matmat(np.asfortranarray(x)), ref[f"{name}/hxh_y"]) < 1e-10
    for t in (tc, tb, ta):
        t.free()


def test_hxh_large_against_dense():
    """A larger product (1D Gaussian x Matern, n = 4096, depth 5) against the
    dense FP64 product.  A and B are compressed to relative tolerance tol per
    block and the product is recompressed with absolute tolerance tol, so the
    error against A (B X) is bounded by about 2 tol (the oracle's own H x H
    lands at 1.3e-10 on this case); recompression alone, measured against
    the product of the two factor trees, stays at rounding level."""
    n, h, tol = 4096, 5, 1e-8
    pts = W.points_1d_sorted(n, seed=3)
    a = W.kernel_matrix(pts, "gaussian", 0.1, 1.0)
    b = W.kernel_matrix(pts, "matern32", 0.2, 1.0)
    ta, tb = Tree.from_dense(a, h, tol), Tree.from_dense(b, h, tol)
    tc = ta.hxh(tb, tol)
    x = np.asfortranarray(np.random.default_rng(0).standard_normal((n, 8)))
    y = tc.matmat(x)
    err = O.rel_fro(y, a @ (b @ x))
    assert err < 2 * tol, err
    y_factors = ta.matmat(tb.matmat(x))
    assert O.rel_fro(y, y_factors) < 1e-12
    for t in (tc, tb, ta):
        t.free()


def _device_recompress(u, v, tol, dense):
    import ctypes as C

    import torch

    from hmat_lib_b200 import abi
    lib = abi.load()
    m, s = u.shape
    n = v.shape[0]
    cap = max(s, min(m, n))
    du = torch.from_numpy(np.asfortranarray(u).T.copy()).cuda()      # column-major m x s
    dv = torch.from_numpy(np.asfortranarray(v).T.copy()).cuda()
    uo = torch.full((cap, m), float("nan"), dtype=torch.float64, device="cuda")
    vo = torch.full((cap, n), float("nan"), dtype=torch.float64, device="cuda")
    rank = C.c_int(-1)
    torch.cuda.synchronize()
    r = lib.hodlr_b200_recompress_dev(m, n, s, C.c_void_p(du.data_ptr()), m,
                                      C.c_void_p(dv.data_ptr()), n, tol, int(dense),
                                      C.c_void_p(uo.data_ptr()), C.c_void_p(vo.data_ptr()),
                                      C.byref(rank), None)
    assert r == abi.SUCCESS, lib.hodlr_b200_last_error()
    k = rank.value
    return uo[:k].cpu().numpy().T, vo[:k].cpu().numpy().T


@pytest.mark.parametrize("c", K.known_answers()["recompress"], ids=lambda c: c["name"])
def test_device_recompress_known_answers(c):
    """hmat_lib's recompression golden values
    (tests/unit_tests/test_hodlr_hodlr_algebra.c:1633-1675 for recompress,
    :1799-1830 for recompress_large_s; absolute truncation at 1e-8) run
    through the device QR + Jacobi routine that multiply_hodlr_hodlr uses:
    same rank, U V^T within hmat_lib's 1e-10, and (recompress) each column
    of U' and V' equal to the golden one up to its sign within 1e-9 -- the
    12-digit values of the 11 x 11 case included."""
    u, v = np.array(c["u"]), np.array(c["v"])
    eu, ev = np.array(c["eu"]), np.array(c["ev"])
    ru, rv = _device_recompress(u, v, 1e-8, c["large"])
    assert ru.shape[1] == eu.shape[1]
    assert np.abs(ru @ rv.T - eu @ ev.T).max() <= K.DELTA
    if not c["large"]:
        for j in range(eu.shape[1]):
            if np.abs(eu[:, j]).max() < 1e-6:
                continue
            sgn = 1.0 if np.dot(ru[:, j], eu[:, j]) >= 0 else -1.0
            assert np.abs(sgn * ru[:, j] - eu[:, j]).max() <= 1e-9
            assert np.abs(sgn * rv[:, j] - ev[:, j]).max() <= 1e-9


def test_hxh_with_int8_subtree_products(lib):
    """Option hxh_precision = 1 runs the subtree products of H x H (depth-
    masked products: leaves and the blocks below each depth) on the int8
    tensor cores: same ranks as the FP64 product within one, and the
    product's action within 1e-10 of the FP64 product's and within 2 tol of
    the dense A (B X)."""
    n, h, tol = 2048, 4, 1e-8
    pts = W.points_1d_sorted(n, seed=3)
    a = W.kernel_matrix(pts, "gaussian", 0.1, 1.0)
    b = W.kernel_matrix(pts, "matern32", 0.2, 1.0)
    ta, tb = Tree.from_dense(a, h, tol), Tree.from_dense(b, h, tol)
    tc64 = ta.hxh(tb, tol)
    lib.hodlr_b200_set_option(b"hxh_precision", 1.0)
    try:
        tcmx = ta.hxh(tb, tol)
    finally:
        lib.hodlr_b200_set_option(b"hxh_precision", 0.0)
    r64 = np.array([u.shape[1] for _, (u, _) in sorted(tc64.data().blocks.items())])
    rmx = np.array([u.shape[1] for _, (u, _) in sorted(tcmx.data().blocks.items())])
    assert int(np.abs(r64 - rmx).max()) <= 1
    x = np.asfortranarray(np.random.default_rng(1).standard_normal((n, 6)))
    y64, ymx = tc64.matmat(x), tcmx.matmat(x)
    assert O.rel_fro(ymx, y64) < 1e-10
    assert O.rel_fro(ymx, a @ (b @ x)) < 2 * tol
    for t in (tcmx, tc64, tb, ta):
        t.free()
