"""Host-side helpers over the hmat_lib tree ABI (library-agnostic).

A tree of height h has internal nodes at depths 0..h-1; node (d, j),
0 <= j < 2**d, covers diagonal leaves [j * 2**(h-d), (j+1) * 2**(h-d)).
Its top-right off-diagonal child is block (d, j, 1) and its bottom-left is
(d, j, 2) -- the same child numbering as hmat_lib
(include/hmat_lib/hodlr.h:186-215).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class TreeData:
    """Plain numpy copy of a HODLR tree."""
    height: int
    leaf_sizes: list
    leaves: list = field(default_factory=list)      # 2**h dense blocks
    blocks: dict = field(default_factory=dict)      # (d, j, c) -> (U, V)

    @property
    def n(self) -> int:
        return int(sum(self.leaf_sizes))

    def node_range(self, d: int, j: int):
        """(offset, size, size of the top-left child) of internal node (d, j)."""
        span = 1 << (self.height - d)
        offs = np.concatenate([[0], np.cumsum(self.leaf_sizes)])
        lo, hi = j * span, (j + 1) * span
        mid = lo + span // 2
        return int(offs[lo]), int(offs[hi] - offs[lo]), int(offs[mid] - offs[lo])

    def ranks(self) -> dict:
        return {k: u.shape[1] for k, (u, v) in self.blocks.items()}

    def to_dense(self) -> np.ndarray:
        n = self.n
        a = np.zeros((n, n))
        off = 0
        for leaf in self.leaves:
            m = leaf.shape[0]
            a[off:off + m, off:off + m] = leaf
            off += m
        for (d, j, c), (u, v) in self.blocks.items():
            o, size, top = self.node_range(d, j)
            if c == 1:
                a[o:o + top, o + top:o + size] = u @ v.T
            else:
                a[o + top:o + size, o:o + top] = u @ v.T
        return a

    def storage(self) -> int:
        """Number of stored doubles: sum m_leaf^2 + sum s (m + n)."""
        w = sum(x.size for x in self.leaves)
        w += sum(u.size + v.size for u, v in self.blocks.values())
        return int(w)


def node_at(tp, d: int, j: int):
    """Internal node (d, j) of a ctypes TreeHODLR pointer."""
    node = tp.contents.root
    for level in range(d - 1, -1, -1):
        bit = (j >> level) & 1
        node = node.contents.children[3 if bit else 0].internal
    return node


def _mat(ptr, m, n) -> np.ndarray:
    if m * n == 0 or not ptr:
        return np.zeros((m, n))
    flat = abi.ptr_array(ptr, m * n)
    return flat.reshape((n, m)).T.copy()      # column-major -> numpy


def walk(tp) -> TreeData:
    """Copy a ctypes tree (from any hmat_lib-ABI library) into TreeData."""
    t = tp.contents
    h = t.height
    leaves, sizes = [], []
    for i in range(1 << h):
        lf = t.innermost_leaves[i].contents.data.diagonal
        sizes.append(lf.m)
        leaves.append(_mat(lf.data, lf.m, lf.m))
    td = TreeData(h, sizes, leaves)
    for d in range(h):
        for j in range(1 << d):
            nd = node_at(tp, d, j).contents
            for c in (1, 2):
                od = nd.children[c].leaf.contents.data.off_diagonal
                td.blocks[(d, j, c)] = (_mat(od.u, od.m, od.s), _mat(od.v, od.n, od.s))
    return td


class HostTreeKeepAlive:
    """Holds the numpy buffers a hand-assembled ctypes tree points into."""

    def __init__(self):
        self.buffers = []

    def fortran(self, a: np.ndarray):
        a = np.asfortranarray(a, dtype=np.float64)
        self.buffers.append(a)
        return a.ctypes.data_as(abi.DP)


def fill_tree(tp, td: TreeData, keep: HostTreeKeepAlive):
    """Point an allocated (empty) ctypes tree at the arrays of `td`.

    Sizes of every node are set as hmat_lib's constructor would set them
    (hmat_lib src/constructors.c:133-176); the data pointers refer to
    buffers kept alive by `keep` (so do NOT free such a tree's data with the
    library's free_tree_data)."""
    t = tp.contents
    h = td.height
    for i in range(1 << h):
        lf = t.innermost_leaves[i].contents.data.diagonal
        lf.m = td.leaf_sizes[i]
        lf.data = keep.fortran(td.leaves[i])
    for d in range(h):
        for j in range(1 << d):
            nd = node_at(tp, d, j).contents
            o, size, top = td.node_range(d, j)
            nd.m = size
            for c in (1, 2):
                u, v = td.blocks[(d, j, c)]
                od = nd.children[c].leaf.contents.data.off_diagonal
                od.m, od.n, od.s = u.shape[0], v.shape[0], u.shape[1]
                od.u = keep.fortran(u)
                od.v = keep.fortran(v)
