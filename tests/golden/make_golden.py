"""Generates the golden fixtures of tests/golden/ (run from the repo root):

    python tests/golden/make_golden.py

known_answers.json -- the hand-derived expectations of hmat_lib's own unit
    tests, rebuilt from their definitions (matrices, block sizes, ranks,
    exact products) plus the few numeric golden values those tests pin
    (each entry cites its source file:line in hmat_lib).
reference_outputs.npz -- outputs of the unmodified reference library
    (oracle/_ref/libhmat_ref.so, built by oracle/Makefile) on seeded kernel
    matrices: ranks of every block, products with seeded right-hand sides,
    and HODLR x HODLR results.

The decay matrices of hmat_lib's constructor tests draw their points with
glibc rand() after srand(42) (tests/unit_tests/test_constructors.c:1077);
the same stream is reproduced here through ctypes and stored.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hmat_lib_b200 import workloads as W  # noqa: E402
from oracle import hodlr_oracle as O, ref_lib  # noqa: E402


def glibc_decay_vectors(m: int, count: int, seed: int = 42):
    """vec[i] = 1 - 2 rand()/RAND_MAX, as fill_decay_matrix_random does
    (hmat_lib tests/utils/common_data.c:129-139), `count` vectors in a row."""
    libc = C.CDLL("libc.so.6")
    libc.srand(C.c_uint(seed))
    RAND_MAX = 2147483647
    out = []
    for _ in range(count):
        out.append([1.0 - 2.0 * (libc.rand() / RAND_MAX) for _ in range(m)])
    return out


def compress_cases():
    """hmat_lib tests/unit_tests/test_constructors.c:725-823: seven blocks
    with their exact rank and factors (signs as LAPACK returns them)."""
    cases = []

    def case(name, m_full, kind, row0, col0, m, n, s, u_idx, v_idx):
        cases.append(dict(name=name, m_full=m_full, kind=kind, row0=row0, col0=col0, m=m, n=n,
                          s=s, u=u_idx, v=v_idx))

    # L_bl: matrix + m (row offset m) -> rows [5, 10), cols [0, 5)
    case("L_bl", 10, "laplacian", 5, 0, 5, 5, 1, {0: 1.0}, {0: -0.0, 4: -1.0})
    case("L_tr", 11, "laplacian", 0, 5, 5, 6, 1, {4: -1.0}, {0: 1.0})
    case("L0.5S_bl", 11, "laplacian_corners_sym", 5, 0, 6, 5, 2, {0: 1.0, 11: -0.5},
         {4: -1.0, 5: -1.0})
    case("L0.5S_tr", 10, "laplacian_corners_sym", 0, 5, 5, 5, 2, {4: 1.0, 5: 0.5},
         {0: -1.0, 9: 1.0})
    case("I", 18, "identity", 5, 0, 5, 4, 1, {}, {0: 1.0})
    case("0", 7, "zeros", 0, 0, 7, 7, 1, {}, {0: 1.0})
    case("L_skew", 13, "laplacian", 9, 0, 4, 9, 1, {0: 1.0}, {8: -1.0})
    return cases


def recompress_cases():
    """hmat_lib tests/unit_tests/test_hodlr_hodlr_algebra.c:1560-1690
    (recompress) and :1755-1790 (recompress_large_s): input factors and the
    expected compressed factors (12-digit golden values for the 11 x 11
    Laplacian-like case)."""
    out = []

    def zeros(ms, ss, ns, big):
        for i, (m, s, n) in enumerate(zip(ms, ss, ns)):
            u = np.zeros((m, s))
            v = np.zeros((n, s))
            eu = np.zeros((m, 1))
            ev = np.zeros((n, 1))
            uf, vf, euf, evf = (x.reshape(-1, order="F") for x in (u, v, eu, ev))
            if i == 0:
                uf[0] = 1; vf[0] = 1; euf[0] = 1; evf[0] = 1
            elif i == 1:
                uf[m - 1] = 1; vf[0] = 1; euf[m - 1] = -1; evf[0] = -1
            elif i == 2:
                uf[0] = 1; vf[n - 1] = 1; euf[0] = 1; evf[n - 1] = 1
            else:
                uf[0] = 1; uf[m] = 1; vf[n - 1] = 1; vf[2 * n - 1] = 1
                euf[0] = 2; evf[n - 1] = 1
            out.append(dict(name=f"zero{i}{'_large' if big else ''}", large=big,
                            u=uf.reshape((m, s), order="F").tolist(),
                            v=vf.reshape((n, s), order="F").tolist(),
                            eu=euf.reshape((m, 1), order="F").tolist(),
                            ev=evf.reshape((n, 1), order="F").tolist()))

    zeros([10, 10, 9, 6], [2, 3, 4, 2], [10, 9, 10, 6], False)
    zeros([10, 10, 9, 6], [10, 9, 9, 12], [10, 9, 10, 6], True)
    for big, s in ((False, 3), (True, 13)):
        m = n = 11
        uf = np.zeros(m * s)
        vf = np.zeros(n * s)
        uf[m - 2] = 2; uf[m - 1] = -4; uf[2 * m - 1] = 1.0; uf[2 * m] = -0.5
        vf[0] = -1; vf[n] = 1.0; vf[n + 1] = -2.0; vf[3 * n - 2] = -2.0; vf[3 * n - 1] = 1.0
        euf = np.zeros(m * 3)
        evf = np.zeros(n * 3)
        euf[m - 2] = 1.887256638321; euf[m - 1] = -5.380155478673; euf[m] = 1.118033988750
        euf[2 * m - 2] = -6.20633538e-17; euf[2 * m] = -3.89445209e-17
        euf[3 * m - 2] = 6.62013882871e-1; euf[3 * m - 1] = 2.32221931143e-1
        evf[0] = -0.943628319160; evf[1] = 0.331006941436
        evf[2 * n - 2] = 0.894427191000; evf[2 * n - 1] = -0.447213595500
        evf[2 * n] = -0.331006941436; evf[2 * n + 1] = -0.943628319160
        out.append(dict(name=f"laplace{'_large' if big else ''}", large=big,
                        u=uf.reshape((m, s), order="F").tolist(),
                        v=vf.reshape((n, s), order="F").tolist(),
                        eu=euf.reshape((m, 3), order="F").tolist(),
                        ev=evf.reshape((n, 3), order="F").tolist()))
    return out


def dense_to_tree_cases():
    """hmat_lib tests/unit_tests/test_constructors.c:1006-1106."""
    ms69 = [None] * 5 + [[29, 40], [21, 10, 5, 33], [10, 11, 1, 9, 5, 20, 7, 6],
                         [2, 8, 7, 4, 1, 5, 4, 2, 3, 10, 5, 6, 5, 2, 3, 2],
                         [1, 1, 5, 3, 2, 5, 2, 2, 1, 1, 4, 2, 2, 1, 1, 2,
                          1, 4, 3, 3, 1, 3, 5, 1, 2, 3, 1, 1, 2, 1, 1, 2]]
    ms155a = [None] * 5 + [[55, 100], [50, 5, 50, 50], [22, 11, 11, 11, 25, 25, 25, 25],
                           [13, 15, 10, 4, 15, 12, 6, 3, 6, 14, 2, 4, 23, 11, 11, 6],
                           [2, 6, 8, 2, 2, 6, 4, 6, 8, 7, 6, 7, 4, 5, 6, 7,
                            8, 4, 2, 3, 7, 4, 5, 2, 4, 4, 3, 6, 2, 9, 2, 4]]
    ms155b = [None] * 5 + [[55, 100], [50, 5, 50, 50], [22, 11, 11, 11, 25, 25, 25, 25],
                           [13, 15, 10, 4, 15, 12, 6, 3, 6, 14, 2, 4, 23, 11, 11, 6],
                           [2, 6, 8, 2, 1, 6, 4, 6, 8, 7, 6, 7, 4, 6, 6, 7,
                            8, 4, 2, 3, 7, 4, 5, 2, 4, 4, 3, 6, 2, 9, 1, 5]]
    cases = []
    for idx in range(10):
        cases.append(dict(name="L0.5S", m=69, height=idx % 5 + 1, ms=ms69[idx], kind="l05s",
                          root_rank=2, other_rank=1))
    # 20 decay matrices drawn in sequence after srand(42): 10 sorted, 10 unsorted
    vecs = glibc_decay_vectors(155, 20)
    for idx in range(20):
        sorted_ = idx < 10
        ms = (ms155a + ms155b)[idx]
        vec = sorted(vecs[idx]) if sorted_ else vecs[idx]
        cases.append(dict(name="DecaySort" if sorted_ else "Decay", m=155,
                          height=idx % 5 + 1, ms=ms, kind="decay", vec=vec,
                          root_rank=1 if sorted_ else 0, other_rank=1 if sorted_ else 0))
    return cases


def main():
    known = dict(compress=compress_cases(), recompress=recompress_cases(),
                 dense_to_tree=dense_to_tree_cases())
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known, f)

    if not ref_lib.available():
        raise SystemExit("reference build missing: make -C oracle")
    out = {}
    cases = [
        ("g21_h3", 21, 3, "gaussian", 0.2, 1.0, 1e-10),
        ("g155_h4", 155, 4, "gaussian", 0.2, 1.0, 1e-10),
        ("m300_h3", 300, 3, "matern32", 0.1, 1e-2, 1e-8),
        ("e517_h4", 517, 4, "exponential", 0.3, 0.0, 1e-8),
        ("g1024_h3", 1024, 3, "gaussian", 0.2, 1.0, 1e-10),
    ]
    for name, n, h, kind, length, diag, tol in cases:
        pts = W.points_1d_sorted(n, seed=7)
        a = W.kernel_matrix(pts, kind, length, diag)
        t = ref_lib.build(a, h, tol)
        td = t.data()
        ranks = np.array([td.blocks[k][0].shape[1] for k in sorted(td.blocks)], dtype=np.int32)
        x = W.rhs(n, 3, seed=11)
        out[f"{name}/ranks"] = ranks
        out[f"{name}/yN"] = ref_lib.multiply_dense(t, x, "N")
        out[f"{name}/yT"] = ref_lib.multiply_dense(t, x, "T")
        out[f"{name}/yL"] = ref_lib.multiply_dense(t, x.T.copy(), "L")
        out[f"{name}/yv"] = ref_lib.multiply_vector(t, x[:, 0].copy())
        if n <= 1024:
            b = W.kernel_matrix(pts, "matern32", 0.2, 1.0)
            tb = ref_lib.build(b, h, tol)
            tc = ref_lib.multiply_hodlr_hodlr(t, tb, 1e-8)
            tdc = tc.data()
            out[f"{name}/hxh_ranks"] = np.array(
                [tdc.blocks[k][0].shape[1] for k in sorted(tdc.blocks)], dtype=np.int32)
            # the product tree applied to x (its dense form is too large to store)
            out[f"{name}/hxh_y"] = O.multiply_dense(tdc, x)
    np.savez_compressed(os.path.join(HERE, "reference_outputs.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
