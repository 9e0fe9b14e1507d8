"""Device parity of dense_to_tree_hodlr (GPU compression) through the C-ABI:
hmat_lib's known answers (ranks exact, reconstruction within its 1e-10
DELTA), ranks and products equal to the reference library's on seeded kernel
matrices, and hmat_lib's input-error behaviour."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, Tree, HodlrError
from oracle import hodlr_oracle as O

import cases as K

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("c", K.known_answers()["dense_to_tree"],
                         ids=lambda c: f"{c['name']}-h{c['height']}-{'ms' if c['ms'] else 'halves'}")
def test_dense_to_tree_known_answers(c):
    """hmat_lib tests/unit_tests/test_constructors.c:1122-1158."""
    a = K.dense_case_matrix(c)
    t = Tree.from_dense(a, c["height"], 1e-8, c["ms"])
    td = t.data()
    if c["ms"] is not None:
        assert td.leaf_sizes == c["ms"]
    assert np.abs(td.to_dense() - a).max() <= K.DELTA
    for (d, j, cc), (u, v) in td.blocks.items():
        want = c["root_rank"] if d == 0 else c["other_rank"]
        if want > 0:
            assert u.shape[1] == want, (d, j, cc)
    t.free()


@pytest.mark.parametrize("c", K.known_answers()["compress"], ids=lambda c: c["name"])
def test_compress_known_answers(c):
    """hmat_lib tests/unit_tests/test_constructors.c:833-946: the block is
    placed as the top-right block of a height-1 tree with leaves [m, n]."""
    blk, eu, ev = K.compress_case_inputs(c)
    a = K.embed_block(blk)
    t = Tree.from_dense(a, 1, 1e-8, [c["m"], c["n"]])
    u, v = t.data().blocks[(0, 0, 1)]
    assert u.shape[1] == c["s"]
    assert np.abs(u @ v.T - eu @ ev.T).max() <= K.DELTA
    assert np.abs(u @ v.T - blk).max() <= K.DELTA
    # V has orthonormal columns, U carries the singular values
    assert np.abs(v.T @ v - np.eye(c["s"])).max() < 1e-12
    t.free()


REF_CASES = [
    ("g21_h3", 21, 3, "gaussian", 0.2, 1.0, 1e-10),
    ("g155_h4", 155, 4, "gaussian", 0.2, 1.0, 1e-10),
    ("m300_h3", 300, 3, "matern32", 0.1, 1e-2, 1e-8),
    ("e517_h4", 517, 4, "exponential", 0.3, 0.0, 1e-8),
    ("g1024_h3", 1024, 3, "gaussian", 0.2, 1.0, 1e-10),
]


@pytest.mark.parametrize("case", REF_CASES, ids=lambda c: c[0])
def test_build_matches_reference(case):
    """Ranks equal the reference's; products agree to rounding."""
    name, n, h, kind, length, diag, tol = case
    ref = K.reference_outputs()
    pts = W.points_1d_sorted(n, seed=7)
    a = W.kernel_matrix(pts, kind, length, diag)
    t = Tree.from_dense(a, h, tol)
    td = t.data()
    ranks = np.array([td.blocks[k][0].shape[1] for k in sorted(td.blocks)])
    np.testing.assert_array_equal(ranks, ref[f"{name}/ranks"])
    x = np.asfortranarray(W.rhs(n, 3, seed=11))
    assert O.rel_fro(t.matmat(x, "N"), ref[f"{name}/yN"]) < 1e-12
    assert O.rel_fro(t.matmat(x, "T"), ref[f"{name}/yT"]) < 1e-12
    assert O.rel_fro(t.matmat(np.asfortranarray(x.T), "L"), ref[f"{name}/yL"]) < 1e-12
    assert O.rel_fro(t.matvec(x[:, 0].copy()), ref[f"{name}/yv"]) < 1e-12
    # the factors are an SVD: V orthonormal, U columns ordered by norm
    for (u, v) in td.blocks.values():
        assert np.abs(v.T @ v - np.eye(v.shape[1])).max() < 1e-10
        nrm = np.linalg.norm(u, axis=0)
        assert np.all(np.diff(nrm) <= 1e-12 * max(nrm[0], 1e-300))
    t.free()


def test_smallest_workload_matvec_against_dense():
    """The n = 1024 Gaussian workload (tol 1e-10, depth 3): H x against the
    dense product."""
    w = W.WORKLOADS["gauss1d_n1024"]
    pts = W.workload_points("gauss1d_n1024")
    a = W.kernel_matrix(pts, w["kind"], w["length"], w["diag"])
    t = Tree.from_dense(a, w["height"], w["tol"])
    x = np.random.default_rng(0).standard_normal(a.shape[0])
    assert O.rel_fro(t.matvec(x), a @ x) < 1e-9
    t.free()


def test_build_input_errors(lib):
    t = Tree(2)
    ierr = C.c_int(-1)
    assert lib.dense_to_tree_hodlr(t.tp, 10, None, None, 1e-8, C.byref(ierr)) == 0
    assert ierr.value == abi.INPUT_ERROR
    a = np.asfortranarray(np.eye(10))
    ms = (C.c_int * 4)(2, 3, 3, 3)   # sums to 11, not 10
    ierr.value = -1
    lib.dense_to_tree_hodlr(t.tp, 10, C.cast(ms, abi.IP), abi.as_dp(a.reshape(-1, order="F")),
                            1e-8, C.byref(ierr))
    assert ierr.value == abi.INPUT_ERROR
    t.free()
    with pytest.raises(HodlrError):
        Tree.from_dense(np.eye(10), 2, 1e-8, [2, 3, 3, 3])


def test_jacobi_sweep_cap_reports_svd_failure(lib):
    """The Jacobi sweep loop is bounded: forcing a cap of one sweep makes a
    non-trivial block report SVD_FAILURE instead of spinning."""
    lib.hodlr_b200_set_option(b"jacobi_max_sweeps", 1.0)
    try:
        pts = W.points_1d_sorted(64, seed=1)
        a = W.kernel_matrix(pts, "gaussian", 0.3, 1.0)
        with pytest.raises(HodlrError) as e:
            Tree.from_dense(a, 1, 1e-12)
        assert e.value.code == abi.SVD_FAILURE
    finally:
        lib.hodlr_b200_set_option(b"jacobi_max_sweeps", 60.0)


def test_sketched_path_known_answers(lib):
    """Force the randomized path for every block wider than 8 columns and
    re-run hmat_lib's dense_to_tree known answers."""
    lib.hodlr_b200_set_option(b"exact_max", 8.0)
    try:
        for c in K.known_answers()["dense_to_tree"]:
            a = K.dense_case_matrix(c)
            t = Tree.from_dense(a, c["height"], 1e-8, c["ms"])
            td = t.data()
            assert np.abs(td.to_dense() - a).max() <= K.DELTA, c["name"]
            for (d, j, cc), (u, v) in td.blocks.items():
                want = c["root_rank"] if d == 0 else c["other_rank"]
                if want > 0:
                    assert u.shape[1] == want, (c["name"], d, j, cc)
            t.free()
    finally:
        lib.hodlr_b200_set_option(b"exact_max", 128.0)


@pytest.mark.parametrize("n,h", [(2048, 4), (4096, 5)])
def test_sketched_build_2d_matern(n, h):
    """The benchmark's kernel family (2D Matern-3/2, l = 0.1, tol 1e-8) at
    sizes the CPU oracle handles: ranks within one of the oracle's dgesdd
    ranks, reconstruction and products within the truncation tolerance."""
    pts = W.points_morton(n, 2, seed=1)
    a = W.kernel_matrix(pts, "matern32", 0.1, 1e-2)
    t = Tree.from_dense(a, h, 1e-8)
    td = t.data()
    ot = O.dense_to_tree(a, h, 1e-8)
    for key, r in ot.ranks().items():
        assert abs(td.ranks()[key] - r) <= 1, (key, td.ranks()[key], r)
    # the truncation error itself is the oracle's (dgesdd at the same tol)
    err_oracle = O.rel_fro(ot.to_dense(), a)
    assert O.rel_fro(td.to_dense(), a) <= 1.25 * err_oracle + 1e-12
    x = np.asfortranarray(np.random.default_rng(3).standard_normal((n, 16)))
    yo = O.multiply_dense(ot, x)
    assert O.rel_fro(t.matmat(x), a @ x) <= 1.25 * O.rel_fro(yo, a @ x) + 1e-12
    assert O.rel_fro(t.matmat(x), yo) < 2e-8
    t.free()


def test_failed_device_builds_release_their_trees(lib):
    """A device build that ends with SVD_FAILURE hands its tree to the caller
    (as dense_to_tree_hodlr does); the Python wrapper frees it before raising,
    so repeated failures do not grow device memory."""
    import torch
    n = 4096
    pts = W.points_morton(n, 2, seed=3)
    a = torch.from_numpy(np.asfortranarray(W.kernel_matrix(pts, "matern32", 0.1, 1e-2))).cuda()
    torch.cuda.synchronize()
    lib.hodlr_b200_set_option(b"sketch_cap", 32.0)
    try:
        def fail_once():
            with pytest.raises(HodlrError) as e:
                DeviceTree.build(a.data_ptr(), n, n, 5, 1e-8)
            assert e.value.code == abi.SVD_FAILURE
            torch.cuda.synchronize()
        fail_once()
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(12):
            fail_once()
        free1 = torch.cuda.mem_get_info()[0]
    finally:
        lib.hodlr_b200_set_option(b"sketch_cap", 0.0)
    # each leaked tree would hold about 5 MB (leaves and factors)
    assert free0 - free1 < 16 * 2 ** 20, (free0, free1)


def test_sketch_growth_bounded_by_memory_budget(lib):
    """A block whose sketch must grow past its starting width (the 3D n = 8192
    exponential workload's top blocks need about 1500 columns, the start is
    256) stops growing when the growth would not fit option sketch_mem_frac
    of the free device memory: SVD_FAILURE with a message naming the option;
    with the default budget the same build succeeds and reaches that width."""
    import torch
    n, h = 8192, 6
    pts = W.points_morton(n, 3, 4)
    d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).cuda()
    lib.hodlr_b200_set_option(b"sketch_mem_frac", 1e-6)
    try:
        with pytest.raises(HodlrError) as e:
            DeviceTree.build_kernel(d_pts.data_ptr(), n, 3, 2, 0.15, 1e-2, h, 1e-8)
        assert e.value.code == abi.SVD_FAILURE
        assert "sketch_mem_frac" in str(e.value)
    finally:
        lib.hodlr_b200_set_option(b"sketch_mem_frac", 0.6)
    t = DeviceTree.build_kernel(d_pts.data_ptr(), n, 3, 2, 0.15, 1e-2, h, 1e-8)
    st = (C.c_double * 18)()
    lib.hodlr_b200_build_stats(st, 18)
    assert st[9] > 1024 and st[4] == 0   # largest sketch, cap hit
    t.free()


@pytest.mark.parametrize("n,h", [(1024, 3), (4096, 5)])
def test_highest_rank_and_workspace_on_built_trees(lib, n, h):
    """get_highest_s is the largest off-diagonal rank of a built tree and
    compute_multiply_hodlr_dense_workspace that rank times the column count
    (hmat_lib src/utils.c:5-26, src/dense_algebra.c:39-44), on trees built by
    dense_to_tree_hodlr."""
    pts = W.points_1d_sorted(n, seed=5)
    a = W.kernel_matrix(pts, "matern32", 0.2, 1e-2)
    t = Tree.from_dense(a, h, 1e-10)
    td = t.data()
    highest = max(u.shape[1] for (u, v) in td.blocks.values())
    assert highest > 1
    assert lib.get_highest_s(t.tp) == highest
    for k in (1, 7, 256):
        assert lib.compute_multiply_hodlr_dense_workspace(t.tp, k) == highest * k
    t.free()
