"""Known-answer cases of hmat_lib's unit tests, rebuilt from their
definitions, shared by the oracle tests (CPU) and the device parity tests."""
from __future__ import annotations

import json
import os

import numpy as np

from hmat_lib_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# |actual - expected| <= DELTA element-wise (hmat_lib tests/utils/expect.h:9
# uses the float literal 1e-10f).
DELTA = float(np.float32(1e-10))


def known_answers():
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def reference_outputs():
    return np.load(os.path.join(GOLDEN, "reference_outputs.npz"))


def matrix_of(kind: str, m: int) -> np.ndarray:
    if kind == "laplacian":
        return W.laplacian(m)
    if kind == "laplacian_corners_sym":
        return W.laplacian_corners(m, True)
    if kind == "identity":
        return np.asfortranarray(np.eye(m))
    if kind == "zeros":
        return np.zeros((m, m), order="F")
    raise ValueError(kind)


def compress_case_inputs(c):
    """(block, expected U, expected V) of a compression known-answer case."""
    a = matrix_of(c["kind"], c["m_full"])
    blk = a[c["row0"]:c["row0"] + c["m"], c["col0"]:c["col0"] + c["n"]]
    eu = np.zeros(c["m"] * c["s"])
    ev = np.zeros(c["n"] * c["s"])
    for k, v in c["u"].items():
        eu[int(k)] = v
    for k, v in c["v"].items():
        ev[int(k)] = v
    return (np.asfortranarray(blk), eu.reshape((c["m"], c["s"]), order="F"),
            ev.reshape((c["n"], c["s"]), order="F"))


def embed_block(blk: np.ndarray) -> np.ndarray:
    """A (m+n) x (m+n) matrix whose top-right block is `blk`, so that a
    height-1 HODLR with leaf sizes [m, n] compresses exactly `blk`."""
    m, n = blk.shape
    a = np.zeros((m + n, m + n), order="F")
    a[:m, m:] = blk
    a[np.arange(m + n), np.arange(m + n)] = 1.0
    return a


def dense_case_matrix(c) -> np.ndarray:
    if c["kind"] == "l05s":
        return W.laplacian_corners(c["m"], True)
    return W.decay_matrix(np.array(c["vec"]), 1.0)


# --- products of hmat_lib tests/unit_tests/test_vector_algebra.c:54-172 and
#     test_hodlr_dense_algebra.c:163-296 (n = 21, tol 0.1, heights 1-3) ---

def laplacian_product_cases(transpose: bool = False):
    """(name, matrix, dense operand, expected H X): Laplacian variants times
    the all-10 matrix have non-zero first / last rows only."""
    m = 21
    out = []
    full = np.full((m, m), 10.0, order="F")
    for name in ("L", "L0.5S", "L0.5A"):
        if name == "L":
            a = W.laplacian(m)
            first, last = 10.0, 10.0
        elif name == "L0.5S":
            a = W.laplacian_corners(m, True)
            first, last = 15.0, 15.0
        else:
            a = W.laplacian_corners(m, False)
            first, last = (15.0, 10.0) if transpose else (10.0, 15.0)
        e = np.zeros((m, m), order="F")
        e[0, :] = first
        e[m - 1, :] = last
        out.append((name, a, full, e))
    eye = np.asfortranarray(np.eye(m))
    for name, x in (("I", eye), ("0", np.zeros((m, m), order="F")), ("L", W.laplacian(m))):
        out.append(("I x " + name, eye, x, x.copy(order="F")))
    return out


def hxh_cases():
    """hmat_lib tests/unit_tests/test_hodlr_hodlr_algebra.c:59-300: exact
    products at n = 21 (tol 1e-8), as (name, A, B, expected A B)."""
    m = 21
    lap = W.laplacian(m)
    conv = W.laplacian_converse(m)
    out = []
    for name, a in (("L", lap), ("L0.5S", W.laplacian_corners(m, True)),
                    ("L0.5A", W.laplacian_corners(m, False))):
        out.append((name + " x LC", a, conv, a @ conv))
    eye = np.eye(m)
    for name, b in (("I", eye), ("0", np.zeros((m, m))), ("L", lap)):
        out.append(("I x " + name, eye, b, b.copy()))
    out.append(("L x L", lap, lap, lap @ lap))
    return out
