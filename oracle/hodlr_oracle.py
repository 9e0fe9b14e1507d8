"""CPU oracle for the HODLR hot path -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of hmat_lib's FP64 algorithms (construction by SVD
compression, HODLR x vector / dense products and their transposes, subtree
products, HODLR x HODLR with QR recompression).  Only tests/, the smoke check
and the CPU-baseline leg of bench.py may import this module, and only as a
checker.  The product (hmat_lib_b200) never imports it.

numpy.linalg.svd calls LAPACK dgesdd, the routine hmat_lib wraps
(hmat_lib src/lapack_wrapper.c:8-59), and numpy.linalg.qr calls dgeqrf; the
reference uses dgeqrt (blocked), whose factors agree with dgeqrf's up to
rounding.  Parity against the real reference is pinned separately in
tests/test_oracle.py by running the reference library built by
oracle/Makefile, and against the hand-derived values of hmat_lib's own unit
tests (tests/golden/).

Trees are hmat_lib_b200.tree.TreeData objects: leaves (2**h dense blocks) and
blocks[(d, j, c)] = (U, V) with c = 1 top-right, c = 2 bottom-left.
"""
from __future__ import annotations

import numpy as np

from hmat_lib_b200.tree import TreeData


# ---------------------------------------------------------------- sizing --

def block_sizes_halves(m: int, height: int) -> list:
    """Leaf sizes when every split gives the top-left child m - m//2
    (hmat_lib src/constructors.c:44-95, split at :60-64)."""
    sizes = [m]
    for _ in range(height):
        nxt = []
        for s in sizes:
            small = s // 2
            nxt += [s - small, small]
        sizes = nxt
    return sizes


# ---------------------------------------------------------- construction --

def truncation_rank_relative(s: np.ndarray, tol: float) -> int:
    """hmat_lib src/constructors.c:329-336: keep index k while
    s[k] >= tol * s[0]; keep at least one; keep exactly one when
    s[0] <= tol (absolute test on the largest value)."""
    k = 1
    if s[0] > tol:
        k = 1
        while k < len(s):
            if s[k] < tol * s[0]:
                break
            k += 1
    return k


def compress_block(a: np.ndarray, tol: float):
    """SVD compression of one off-diagonal block
    (hmat_lib src/constructors.c:308-367): U is scaled by the kept singular
    values (:344-348), V is stored untransposed (:356-360)."""
    u, s, vt = np.linalg.svd(a, full_matrices=False)
    k = truncation_rank_relative(s, tol)
    return u[:, :k] * s[:k], vt[:k, :].T.copy()


def dense_to_tree(a: np.ndarray, height: int, tol: float, ms=None) -> TreeData:
    """hmat_lib src/constructors.c:629-704 (dense_to_tree_hodlr)."""
    m = a.shape[0]
    sizes = list(ms) if ms is not None else block_sizes_halves(m, height)
    if sum(sizes) != m:
        raise ValueError("INPUT_ERROR: block sizes do not sum to m")
    td = TreeData(height, sizes)
    off = 0
    for s in sizes:                                   # copy_diagonal_blocks
        td.leaves.append(a[off:off + s, off:off + s].copy())
        off += s
    for d in range(height):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            td.blocks[(d, j, 1)] = compress_block(a[o:o + top, o + top:o + size], tol)
            td.blocks[(d, j, 2)] = compress_block(a[o + top:o + size, o:o + top], tol)
    return td


# ------------------------------------------------------------- products --

def multiply_dense(td: TreeData, x: np.ndarray) -> np.ndarray:
    """Y = H X (hmat_lib src/dense_algebra.c:361-429; k = 1 is
    multiply_vector, src/vector_algebra.c:131-197).  Leaves first with
    beta = 0, then every off-diagonal block adds U (V^T X[cols])."""
    vec = x.ndim == 1
    x2 = x.reshape(x.shape[0], -1)
    y = np.zeros_like(x2)
    off = 0
    for leaf in td.leaves:
        mm = leaf.shape[0]
        y[off:off + mm] = leaf @ x2[off:off + mm]
        off += mm
    for d in range(td.height - 1, -1, -1):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            u, v = td.blocks[(d, j, 1)]
            y[o:o + top] += u @ (v.T @ x2[o + top:o + size])
            u, v = td.blocks[(d, j, 2)]
            y[o + top:o + size] += u @ (v.T @ x2[o:o + top])
    return y[:, 0] if vec else y


def multiply_transpose_dense(td: TreeData, x: np.ndarray) -> np.ndarray:
    """Y = H^T X (hmat_lib src/dense_algebra.c:617-771): leaves D^T, and
    block (d, j, 2)^T lands in the top rows, (d, j, 1)^T in the bottom."""
    y = np.zeros_like(x)
    off = 0
    for leaf in td.leaves:
        mm = leaf.shape[0]
        y[off:off + mm] = leaf.T @ x[off:off + mm]
        off += mm
    for d in range(td.height):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            u, v = td.blocks[(d, j, 2)]
            y[o:o + top] += v @ (u.T @ x[o + top:o + size])
            u, v = td.blocks[(d, j, 1)]
            y[o + top:o + size] += v @ (u.T @ x[o:o + top])
    return y


def multiply_dense_hodlr(td: TreeData, x: np.ndarray) -> np.ndarray:
    """Y = X H, X is k x n (hmat_lib src/dense_algebra.c:957-1026)."""
    y = np.zeros_like(x)
    off = 0
    for leaf in td.leaves:
        mm = leaf.shape[0]
        y[:, off:off + mm] = x[:, off:off + mm] @ leaf
        off += mm
    for d in range(td.height):
        for j in range(1 << d):
            o, size, top = td.node_range(d, j)
            u, v = td.blocks[(d, j, 1)]
            y[:, o + top:o + size] += (x[:, o:o + top] @ u) @ v.T
            u, v = td.blocks[(d, j, 2)]
            y[:, o:o + top] += (x[:, o + top:o + size] @ u) @ v.T
    return y


def subtree(td: TreeData, d: int, j: int) -> TreeData:
    """The HODLR rooted at internal node (d, j) (the operand of
    hmat_lib's multiply_internal_node_* functions, src/dense_algebra.c:492,
    710, 1087)."""
    h = td.height - d
    span = 1 << h
    sub = TreeData(h, td.leaf_sizes[j * span:(j + 1) * span],
                   td.leaves[j * span:(j + 1) * span])
    for dd in range(h):
        for jj in range(1 << dd):
            for c in (1, 2):
                sub.blocks[(dd, jj, c)] = td.blocks[(d + dd, (j << dd) + jj, c)]
    return sub


# ----------------------------------------------------- recompression ----

def truncation_rank_absolute(s: np.ndarray, tol: float) -> int:
    """hmat_lib src/hodlr_algebra.c:160-163 and :305-308: stop at the first
    k >= 1 with s[k] <= tol (an ABSOLUTE threshold, whatever the doc comment
    at :32-37 says); at least one value is kept."""
    k = 1
    while k < len(s):
        if s[k] <= tol:
            break
        k += 1
    return k


def recompress(u: np.ndarray, v: np.ndarray, tol: float):
    """hmat_lib src/hodlr_algebra.c:97-211: QR of U and V, SVD of
    R_U R_V^T, absolute truncation, U <- Q_U W Sigma, V <- Q_V Z."""
    qu, ru = np.linalg.qr(u)
    qv, rv = np.linalg.qr(v)
    w, s, zt = np.linalg.svd(ru @ rv.T)
    k = truncation_rank_absolute(s, tol)
    return qu @ (w[:, :k] * s[:k]), qv @ zt[:k].T


def recompress_large_s(u: np.ndarray, v: np.ndarray, tol: float):
    """hmat_lib src/hodlr_algebra.c:280-343: dense U V^T, then a full SVD
    with min(m, n) values and absolute truncation."""
    a = u @ v.T
    w, s, zt = np.linalg.svd(a, full_matrices=False)
    k = truncation_rank_absolute(s, tol)
    return w[:, :k] * s[:k], zt[:k].T.copy()


def recompress_auto(u, v, tol):
    """Path choice of hmat_lib src/hodlr_algebra.c:406-419."""
    if u.shape[1] < min(u.shape[0], v.shape[0]):
        return recompress(u, v, tol)
    return recompress_large_s(u, v, tol)


# ------------------------------------------------------ HODLR x HODLR ---

def _ancestor_terms(t1: TreeData, t2: TreeData, d: int, j: int, rows, cols):
    """Low-rank terms of (H1 H2)[rows, cols] that pass through ancestors of
    node (d, j): for each ancestor, the row band of H1's off-diagonal block
    times the column band of H2's mirrored block
    (hmat_lib src/hodlr_algebra.c:467-540)."""
    us, vs = [], []
    jj = j
    for dd in range(d - 1, -1, -1):
        child = jj & 1
        jj >>= 1
        o, size, top = t1.node_range(dd, jj)
        if child == 0:          # node lies in the top half: H1 top-right x H2 bottom-left
            u1, v1 = t1.blocks[(dd, jj, 1)]
            u2, v2 = t2.blocks[(dd, jj, 2)]
            r0 = o
            c0 = o
        else:                   # bottom half: H1 bottom-left x H2 top-right
            u1, v1 = t1.blocks[(dd, jj, 2)]
            u2, v2 = t2.blocks[(dd, jj, 1)]
            r0 = o + top
            c0 = o + top
        core = v1.T @ u2                              # s1 x s2
        us.append(u1[rows[0] - r0:rows[1] - r0])
        vs.append(v2[cols[0] - c0:cols[1] - c0] @ core.T)
    return us, vs


def multiply_hodlr_hodlr(t1: TreeData, t2: TreeData, tol: float) -> TreeData:
    """out = H1 H2 (hmat_lib src/hodlr_algebra.c:1452-1553).

    Diagonal leaves: D1 D2 plus every ancestor's low-rank contribution
    restricted to the leaf (:1267-1333, :1189-1211).  Off-diagonal block of
    node (d, j): the ancestor terms (:467-540), then the two in-node terms
    [H1_TL U2 | U1] and [V2 | H2_BR^T V1] (top-right; :670-705 at the leaf
    level, :930-966 above it), recompressed (:406-419)."""
    h = t1.height
    out = TreeData(h, list(t1.leaf_sizes))
    nleaf = 1 << h
    offs = np.concatenate([[0], np.cumsum(t1.leaf_sizes)])
    for i in range(nleaf):
        r = (int(offs[i]), int(offs[i + 1]))
        dd = t1.leaves[i] @ t2.leaves[i]
        us, vs = _ancestor_terms(t1, t2, h, i, r, r)
        for u, v in zip(us, vs):
            dd = dd + u @ v.T
        out.leaves.append(dd)
    for d in range(h):
        for j in range(1 << d):
            o, size, top = t1.node_range(d, j)
            left = subtree(t1, d + 1, 2 * j) if d + 1 < h else None
            right = subtree(t1, d + 1, 2 * j + 1) if d + 1 < h else None
            left2 = subtree(t2, d + 1, 2 * j) if d + 1 < h else None
            right2 = subtree(t2, d + 1, 2 * j + 1) if d + 1 < h else None
            # top-right block: rows [o, o+top), cols [o+top, o+size)
            u1, v1 = t1.blocks[(d, j, 1)]
            u2, v2 = t2.blocks[(d, j, 1)]
            us, vs = _ancestor_terms(t1, t2, d, j, (o, o + top), (o + top, o + size))
            if left is None:
                h1_tl_u2 = t1.leaves[2 * j] @ u2
                h2_br_v1 = t2.leaves[2 * j + 1].T @ v1
            else:
                h1_tl_u2 = multiply_dense(left, u2)
                h2_br_v1 = multiply_transpose_dense(right2, v1)
            us += [h1_tl_u2, u1]
            vs += [v2, h2_br_v1]
            out.blocks[(d, j, 1)] = recompress_auto(np.hstack(us), np.hstack(vs), tol)
            # bottom-left block: rows [o+top, o+size), cols [o, o+top)
            u1, v1 = t1.blocks[(d, j, 2)]
            u2, v2 = t2.blocks[(d, j, 2)]
            us, vs = _ancestor_terms(t1, t2, d, j, (o + top, o + size), (o, o + top))
            if left is None:
                h1_br_u2 = t1.leaves[2 * j + 1] @ u2
                h2_tl_v1 = t2.leaves[2 * j].T @ v1
            else:
                h1_br_u2 = multiply_dense(right, u2)
                h2_tl_v1 = multiply_transpose_dense(left2, v1)
            us += [h1_br_u2, u1]
            vs += [v2, h2_tl_v1]
            out.blocks[(d, j, 2)] = recompress_auto(np.hstack(us), np.hstack(vs), tol)
    return out


# ---------------------------------------------------------- workloads ---

def rel_fro(a, b) -> float:
    """||a - b||_F / ||b||_F (0 when both vanish)."""
    nb = np.linalg.norm(b)
    na = np.linalg.norm(a - b)
    return float(na / nb) if nb > 0 else float(na)
