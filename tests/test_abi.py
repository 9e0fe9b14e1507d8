"""C-ABI boundary checks that need no GPU: the library loads, exports every
function declared in include/hmat_lib/*.h, its structs have the header's
layout, and the host-only tree skeleton functions behave like hmat_lib's
(hmat_lib src/allocators.c, tests/unit_tests/test_allocators.c)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from hmat_lib_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(INCLUDE, "hmat_lib")):
        text = open(os.path.join(INCLUDE, "hmat_lib", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name in ("if", "sizeof", "defined", "void", "int", "double", "char", "size_t"):
                continue
            names.add(name)
    return names


def test_library_exports_every_declared_function(lib):
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_layout_matches_header():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "hmat_lib/hodlr.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(struct NodeDiagonal), sizeof(struct NodeOffDiagonal),
         sizeof(struct HODLRLeafNode), sizeof(struct HODLRInternalNode), sizeof(struct TreeHODLR),
         offsetof(struct HODLRLeafNode, parent));
  printf("%zu %zu %zu\n", offsetof(struct NodeOffDiagonal, s), offsetof(struct TreeHODLR, len_work_queue),
         offsetof(struct HODLRInternalNode, m));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "p")
        subprocess.check_call(["gcc", "-I", INCLUDE, c, "-o", exe])
        out = subprocess.check_output([exe]).decode().split()
    got = [C.sizeof(abi.NodeDiagonal), C.sizeof(abi.NodeOffDiagonal), C.sizeof(abi.HODLRLeafNode),
           C.sizeof(abi.HODLRInternalNode), C.sizeof(abi.TreeHODLR), abi.HODLRLeafNode.parent.offset,
           abi.NodeOffDiagonal.s.offset, abi.TreeHODLR.len_work_queue.offset,
           abi.HODLRInternalNode.m.offset]
    assert [int(x) for x in out] == got


@pytest.mark.parametrize("height", [1, 2, 3, 5, 8])
def test_array_sizes(lib, height):
    """hmat_lib src/allocators.c:499-512: 2^h - 1 internal nodes,
    6 * 2^(h-1) - 2 leaves, 2^(h-1) queue entries, 2^h innermost leaves."""
    si, sl, sq, sil = (C.c_size_t() for _ in range(4))
    lib.compute_construct_tree_array_sizes(height, C.byref(si), C.byref(sl), C.byref(sq), C.byref(sil))
    n = 2 ** (height - 1)
    assert si.value == (2 * n - 1) * C.sizeof(abi.HODLRInternalNode)
    assert sl.value == (6 * n - 2) * C.sizeof(abi.HODLRLeafNode)
    assert sq.value == n * C.sizeof(C.c_void_p)
    assert sil.value == 2 * n * C.sizeof(C.c_void_p)


def _check_tree(tp, height):
    t = tp.contents
    assert t.height == height
    assert t.len_work_queue == 2 ** (height - 1)
    assert not t.root.contents.parent
    # every internal node links back to its parent; leaves are typed and empty
    stack = [(t.root, 0)]
    n_internal = 0
    while stack:
        node, d = stack.pop()
        n_internal += 1
        nd = node.contents
        for c in (1, 2):
            leaf = nd.children[c].leaf.contents
            assert leaf.type == abi.OFFDIAGONAL
            assert C.addressof(leaf.parent.contents) == C.addressof(nd)
            od = leaf.data.off_diagonal
            assert (od.m, od.s, od.n) == (0, 0, 0) and not od.u and not od.v
        if d == height - 1:
            for c in (0, 3):
                leaf = nd.children[c].leaf.contents
                assert leaf.type == abi.DIAGONAL and leaf.data.diagonal.m == 0
        else:
            for c in (0, 3):
                ch = nd.children[c].internal
                assert C.addressof(ch.contents.parent.contents) == C.addressof(nd)
                stack.append((ch, d + 1))
    assert n_internal == 2 ** height - 1
    # innermost leaves in order, work queue = their parents
    for i in range(2 ** height):
        leaf = t.innermost_leaves[i].contents
        parent = t.work_queue[i // 2].contents
        child = parent.children[3 if i % 2 else 0].leaf.contents
        assert C.addressof(child) == C.addressof(leaf)


@pytest.mark.parametrize("height", [1, 2, 4, 7])
@pytest.mark.parametrize("fn", ["allocate_tree", "allocate_tree_monolithic"])
def test_allocate_and_free(lib, height, fn):
    ierr = C.c_int(-1)
    tp = getattr(lib, fn)(height, C.byref(ierr))
    assert ierr.value == abi.SUCCESS
    _check_tree(tp, height)
    assert (bool(tp.contents.memory_leaf_ptr) == (fn == "allocate_tree_monolithic"))
    assert lib.get_highest_s(tp) == 0
    lib.free_tree_hodlr(C.byref(tp))
    assert not tp


@pytest.mark.parametrize("fn", ["allocate_tree", "allocate_tree_monolithic"])
def test_allocate_bad_height(lib, fn):
    ierr = C.c_int(-1)
    tp = getattr(lib, fn)(0, C.byref(ierr))
    assert not tp and ierr.value == abi.INPUT_ERROR


def test_construct_tree_from_caller_arrays(lib):
    h = 3
    si, sl, sq, sil = (C.c_size_t() for _ in range(4))
    lib.compute_construct_tree_array_sizes(h, C.byref(si), C.byref(sl), C.byref(sq), C.byref(sil))
    bufs = [C.create_string_buffer(x.value) for x in (si, sl, sq, sil)]
    tree = abi.TreeHODLR()
    ierr = C.c_int(-1)
    lib.construct_tree(h, C.byref(tree), C.cast(bufs[0], abi.INP),
                       C.cast(bufs[1], C.POINTER(abi.HODLRLeafNode)),
                       C.cast(bufs[2], C.POINTER(abi.INP)),
                       C.cast(bufs[3], C.POINTER(C.POINTER(abi.HODLRLeafNode))), C.byref(ierr))
    assert ierr.value == abi.SUCCESS
    _check_tree(C.pointer(tree), h)


def test_free_null_is_noop(lib):
    lib.free_tree_hodlr(None)
    tp = abi.TP()
    lib.free_tree_hodlr(C.byref(tp))
    lib.free_tree_data(None)


def test_allocation_failure_is_reported(lib):
    """The host-allocator seam plays the role of hmat_lib's _TEST_HODLR
    malloc injection (tests/utils/expect.h:3-5, test_allocators.c:46-100):
    a failing allocation yields ALLOCATION_FAILURE and no leak/crash."""
    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    libc.free.argtypes = [C.c_void_p]
    ALLOC = C.CFUNCTYPE(C.c_void_p, C.c_size_t)
    FREE = C.CFUNCTYPE(None, C.c_void_p)
    cases = [("allocate_tree_monolithic", k) for k in range(5)] + \
        [("allocate_tree", k) for k in range(0, 32, 3)]
    for fn, fail_at in cases:
        count = [0]

        def alloc(n, count=count, fail_at=fail_at):
            count[0] += 1
            if count[0] == fail_at + 1:
                return None
            return libc.malloc(n)

        a, f = ALLOC(alloc), FREE(lambda p: libc.free(p))
        lib.hodlr_b200_set_host_allocator(C.cast(a, C.c_void_p), C.cast(f, C.c_void_p))
        try:
            ierr = C.c_int(-1)
            tp = getattr(lib, fn)(3, C.byref(ierr))
            assert ierr.value == abi.ALLOCATION_FAILURE and not tp, (fn, fail_at)
        finally:
            lib.hodlr_b200_set_host_allocator(None, None)
