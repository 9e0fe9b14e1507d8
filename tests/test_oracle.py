"""Pins the CPU oracle (oracle/hodlr_oracle.py) before it is trusted as the
checker of the device path: against the known answers of hmat_lib's unit
tests (tests/golden/known_answers.json), against outputs of the unmodified
reference library stored in tests/golden/reference_outputs.npz, and -- when
oracle/_ref/libhmat_ref.so is present -- against fresh reference runs."""
import numpy as np
import pytest

from hmat_lib_b200 import workloads as W
from oracle import hodlr_oracle as O
from oracle import ref_lib

import cases as K


def _uvt(u, v):
    return u @ v.T


@pytest.mark.parametrize("c", K.known_answers()["compress"], ids=lambda c: c["name"])
def test_oracle_compress_known_answers(c):
    """hmat_lib tests/unit_tests/test_constructors.c:833-873 (rank, U, V) and
    :884-946 (reconstruction)."""
    blk, eu, ev = K.compress_case_inputs(c)
    u, v = O.compress_block(blk, 1e-8)
    assert u.shape[1] == c["s"]
    assert np.abs(_uvt(u, v) - _uvt(eu, ev)).max() <= K.DELTA
    # factors equal up to the sign of each singular pair
    for j in range(c["s"]):
        sgn = 1.0 if np.dot(u[:, j], eu[:, j]) + np.dot(v[:, j], ev[:, j]) >= 0 else -1.0
        assert np.abs(sgn * u[:, j] - eu[:, j]).max() <= K.DELTA
        assert np.abs(sgn * v[:, j] - ev[:, j]).max() <= K.DELTA
    assert np.abs(_uvt(u, v) - blk).max() <= K.DELTA


@pytest.mark.parametrize("c", K.known_answers()["recompress"], ids=lambda c: c["name"])
def test_oracle_recompress_known_answers(c):
    """hmat_lib tests/unit_tests/test_hodlr_hodlr_algebra.c:1725-1750 and
    :1799-1830 (absolute truncation at 1e-8)."""
    u, v = np.array(c["u"]), np.array(c["v"])
    eu, ev = np.array(c["eu"]), np.array(c["ev"])
    fn = O.recompress_large_s if c["large"] else O.recompress
    ru, rv = fn(u, v, 1e-8)
    assert ru.shape[1] == eu.shape[1]
    assert np.abs(_uvt(ru, rv) - _uvt(eu, ev)).max() <= K.DELTA
    if not c["large"]:
        for j in range(eu.shape[1]):
            if np.abs(eu[:, j]).max() < 1e-6:
                continue
            sgn = 1.0 if np.dot(ru[:, j], eu[:, j]) >= 0 else -1.0
            assert np.abs(sgn * ru[:, j] - eu[:, j]).max() <= 1e-9
            assert np.abs(sgn * rv[:, j] - ev[:, j]).max() <= 1e-9


@pytest.mark.parametrize("c", K.known_answers()["dense_to_tree"],
                         ids=lambda c: f"{c['name']}-h{c['height']}-{'ms' if c['ms'] else 'halves'}")
def test_oracle_dense_to_tree_known_answers(c):
    """hmat_lib tests/unit_tests/test_constructors.c:1122-1158."""
    a = K.dense_case_matrix(c)
    td = O.dense_to_tree(a, c["height"], 1e-8, c["ms"])
    assert np.abs(td.to_dense() - a).max() <= K.DELTA
    for (d, j, cc), (u, v) in td.blocks.items():
        want = c["root_rank"] if d == 0 else c["other_rank"]
        if want > 0:
            assert u.shape[1] == want, (d, j, cc)


@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("height", [1, 2, 3])
def test_oracle_product_known_answers(height, transpose):
    """hmat_lib tests/unit_tests/test_hodlr_dense_algebra.c:307-430 and
    test_vector_algebra.c:184-215."""
    for name, a, x, e in K.laplacian_product_cases(transpose):
        td = O.dense_to_tree(a, height, 0.1)
        y = O.multiply_transpose_dense(td, x) if transpose else O.multiply_dense(td, x)
        assert np.abs(y - e).max() <= K.DELTA, name
        yv = O.multiply_dense(td, x[:, 0]) if not transpose else None
        if yv is not None:
            assert np.abs(yv - e[:, 0]).max() <= K.DELTA, name


@pytest.mark.parametrize("height", [1, 2, 3])
def test_oracle_hxh_known_answers(height):
    for name, a, b, e in K.hxh_cases():
        ta = O.dense_to_tree(a, height, 1e-8)
        tb = O.dense_to_tree(b, height, 1e-8)
        tc = O.multiply_hodlr_hodlr(ta, tb, 1e-8)
        assert np.abs(tc.to_dense() - e).max() <= K.DELTA, name


REF_CASES = [
    ("g21_h3", 21, 3, "gaussian", 0.2, 1.0, 1e-10),
    ("g155_h4", 155, 4, "gaussian", 0.2, 1.0, 1e-10),
    ("m300_h3", 300, 3, "matern32", 0.1, 1e-2, 1e-8),
    ("e517_h4", 517, 4, "exponential", 0.3, 0.0, 1e-8),
    ("g1024_h3", 1024, 3, "gaussian", 0.2, 1.0, 1e-10),
]


@pytest.mark.parametrize("case", REF_CASES, ids=lambda c: c[0])
def test_oracle_matches_reference_fixtures(case):
    name, n, h, kind, length, diag, tol = case
    ref = K.reference_outputs()
    pts = W.points_1d_sorted(n, seed=7)
    a = W.kernel_matrix(pts, kind, length, diag)
    td = O.dense_to_tree(a, h, tol)
    ranks = np.array([td.blocks[k][0].shape[1] for k in sorted(td.blocks)])
    np.testing.assert_array_equal(ranks, ref[f"{name}/ranks"])
    x = W.rhs(n, 3, seed=11)
    assert O.rel_fro(O.multiply_dense(td, x), ref[f"{name}/yN"]) < 1e-13
    assert O.rel_fro(O.multiply_transpose_dense(td, x), ref[f"{name}/yT"]) < 1e-13
    assert O.rel_fro(O.multiply_dense_hodlr(td, x.T.copy()), ref[f"{name}/yL"]) < 1e-13
    assert O.rel_fro(O.multiply_dense(td, x[:, 0]), ref[f"{name}/yv"]) < 1e-13
    b = W.kernel_matrix(pts, "matern32", 0.2, 1.0)
    tc = O.multiply_hodlr_hodlr(td, O.dense_to_tree(b, h, tol), 1e-8)
    rc = np.array([tc.blocks[k][0].shape[1] for k in sorted(tc.blocks)])
    np.testing.assert_array_equal(rc, ref[f"{name}/hxh_ranks"])
    assert O.rel_fro(O.multiply_dense(tc, x), ref[f"{name}/hxh_y"]) < 1e-12


@pytest.mark.skipif(not ref_lib.available(), reason="reference build absent")
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_matches_reference_library(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(40, 400))
    h = int(rng.integers(1, 5))
    pts = W.points_1d_sorted(n, seed=seed)
    a = W.kernel_matrix(pts, "exponential", float(rng.uniform(0.05, 0.5)), 0.5)
    ms = None
    if seed == 2:
        ms = list(rng.multinomial(n - 2 ** h, np.ones(2 ** h) / 2 ** h) + 1)
    rt = ref_lib.build(a, h, 1e-9, ms)
    td = O.dense_to_tree(a, h, 1e-9, ms)
    rd = rt.data()
    assert td.ranks() == rd.ranks()
    assert O.rel_fro(td.to_dense(), rd.to_dense()) < 1e-13
    x = rng.standard_normal((n, 4))
    assert O.rel_fro(O.multiply_dense(td, x), ref_lib.multiply_dense(rt, x)) < 1e-13


# ---- rank-model oracle (pins oracle/rank_mlp_oracle.py) --------------------------

def test_rank_mlp_oracle_gradient_matches_finite_differences():
    """Central differences of the oracle's loss against its analytic
    gradient, on every trainable entry class (W1, b1, W2, b2, W3, b3)."""
    from oracle import rank_mlp_oracle as R
    rng = np.random.default_rng(3)
    x = rng.standard_normal((40, R.IN)) * 2.0 + 1.0
    t = rng.standard_normal(40)
    p = R.random_params(rng, x)
    _, g = R.loss_and_gradient(p, x, t)
    picks = list(rng.choice(np.arange(R.W1, R.B1), 6)) + list(rng.choice(np.arange(R.B1, R.W2), 4)) \
        + list(rng.choice(np.arange(R.W2, R.B2), 10)) + list(rng.choice(np.arange(R.B2, R.W3), 4)) \
        + list(rng.choice(np.arange(R.W3, R.B3), 4)) + [R.B3]
    for i in picks:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (R.loss_and_gradient(pp, x, t)[0] - R.loss_and_gradient(pm, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])
    assert np.all(g[:R.NORM] == 0.0)


def test_rank_mlp_oracle_adam_matches_formula():
    from oracle import rank_mlp_oracle as R
    rng = np.random.default_rng(4)
    p = R.random_params(rng)
    g = rng.standard_normal(R.SIZE)
    m = np.zeros(R.SIZE)
    v = np.zeros(R.SIZE)
    p1, m1, v1 = R.adam_step(p, g, m, v, 1, 1e-2)
    # first Adam step moves every trainable entry by lr |g| / (|g| + eps)
    d = (p - p1)[R.NORM:]
    ga = np.abs(g[R.NORM:])
    assert np.allclose(np.abs(d), 1e-2 * ga / (ga + 1e-8), rtol=1e-9)
    assert np.all(np.sign(d) == np.sign(g[R.NORM:]))
    assert np.array_equal(p1[:R.NORM], p[:R.NORM])
