"""Device parity of multiply_hodlr_hodlr (HODLR x HODLR with recompression)
through the C-ABI: hmat_lib's known answers
(tests/unit_tests/test_hodlr_hodlr_algebra.c:59-338: exact products at
n = 21, tol 1e-8, element-wise within its 1e-10 DELTA, ranks equal to the
expected tree's) and the reference library's ranks and products on seeded
kernel matrices (tests/golden/reference_outputs.npz)."""
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
    dense FP64 product: error of the order of the recompression tolerance."""
    n, h = 4096, 5
    pts = W.points_1d_sorted(n, seed=3)
    a = W.kernel_matrix(pts, "gaussian", 0.1, 1.0)
    b = W.kernel_matrix(pts, "matern32", 0.2, 1.0)
    ta, tb = Tree.from_dense(a, h, 1e-8), Tree.from_dense(b, h, 1e-8)
    tc = ta.hxh(tb, 1e-8)
    x = np.asfortranarray(np.random.default_rng(0).standard_normal((n, 8)))
    err = O.rel_fro(tc.matmat(x), a @ (b @ x))
    assert err < 1e-7, err
    oc = O.multiply_hodlr_hodlr(O.dense_to_tree(a, h, 1e-8), O.dense_to_tree(b, h, 1e-8), 1e-8)
    assert O.rel_fro(tc.matmat(x), O.multiply_dense(oc, x)) < 1e-7
    for t in (tc, tb, ta):
        t.free()
