"""Python mirror of the hmat_lib C interface, calling libhodlr_b200.so.

Each method maps to one C entry point with hmat_lib's argument meaning and
error behaviour (a non-SUCCESS ierr raises HodlrError carrying the code).
Used by the parity tests and the benchmark; C callers link the library
directly (include/hmat_lib/*.h).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .tree import TreeData, walk, fill_tree, HostTreeKeepAlive


class HodlrError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str = ""):
        self.code = code
        super().__init__(f"{where}: {abi.ERROR_NAMES.get(code, code)} {msg}".strip())


def lib():
    return abi.load()


def _check(ierr: C.c_int, where: str):
    if ierr.value != abi.SUCCESS:
        raise HodlrError(ierr.value, where, lib().hodlr_b200_last_error().decode())


class Tree:
    """A TreeHODLR allocated by libhodlr_b200 (allocate_tree_monolithic)."""

    def __init__(self, height: int, piecewise: bool = False):
        ierr = C.c_int(0)
        fn = lib().allocate_tree if piecewise else lib().allocate_tree_monolithic
        self.tp = fn(height, C.byref(ierr))
        _check(ierr, "allocate_tree")
        self.height = height
        self.keep = None          # numpy buffers of a hand-assembled tree
        self.owns_data = False

    # -- construction ------------------------------------------------------
    @classmethod
    def from_dense(cls, a: np.ndarray, height: int, tol: float, ms=None) -> "Tree":
        """dense_to_tree_hodlr (hmat_lib src/constructors.c:629)."""
        t = cls(height)
        a = np.asfortranarray(a, dtype=np.float64)
        ierr = C.c_int(0)
        msp = None
        if ms is not None:
            arr = (C.c_int * len(ms))(*ms)
            msp = C.cast(arr, abi.IP)
        res = lib().dense_to_tree_hodlr(t.tp, a.shape[0], msp,
                                        a.ctypes.data_as(abi.DP), tol, C.byref(ierr))
        t.owns_data = True
        if ierr.value != abi.SUCCESS:
            code = ierr.value
            t.free()
            raise HodlrError(code, f"dense_to_tree_hodlr (info {res})",
                             lib().hodlr_b200_last_error().decode())
        return t

    @classmethod
    def from_tree_data(cls, td: TreeData) -> "Tree":
        """A caller-assembled tree pointing at numpy buffers."""
        t = cls(td.height)
        t.keep = HostTreeKeepAlive()
        fill_tree(t.tp, td, t.keep)
        return t

    # -- products ----------------------------------------------------------
    def matvec(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.empty_like(x)
        ierr = C.c_int(0)
        lib().multiply_vector(self.tp, abi.as_dp(x), abi.as_dp(out), C.byref(ierr))
        _check(ierr, "multiply_vector")
        return out

    def matmat(self, x: np.ndarray, op: str = "N") -> np.ndarray:
        """op N: H X, T: H^T X, L: X H (X is k x n)."""
        x = np.asfortranarray(x, dtype=np.float64)
        out = np.zeros_like(x, order="F")
        ierr = C.c_int(0)
        xp, op_ = x.ctypes.data_as(abi.DP), out.ctypes.data_as(abi.DP)
        ld = max(x.shape[0], 1)
        if op == "N":
            lib().multiply_hodlr_dense(self.tp, xp, x.shape[1], ld, op_, ld, C.byref(ierr))
        elif op == "T":
            lib().multiply_hodlr_transpose_dense(self.tp, xp, x.shape[1], ld, op_, ld,
                                                 C.byref(ierr))
        elif op == "L":
            lib().multiply_dense_hodlr(self.tp, xp, x.shape[0], ld, op_, ld, C.byref(ierr))
        else:
            raise ValueError(op)
        _check(ierr, f"multiply ({op})")
        return out

    def hxh(self, other: "Tree", tol: float) -> "Tree":
        out = Tree(self.height)
        ierr = C.c_int(0)
        lib().multiply_hodlr_hodlr(self.tp, other.tp, out.tp, tol, C.byref(ierr))
        out.owns_data = True
        if ierr.value != abi.SUCCESS:
            code = ierr.value
            out.free()
            raise HodlrError(code, "multiply_hodlr_hodlr", lib().hodlr_b200_last_error().decode())
        return out

    # -- inspection --------------------------------------------------------
    def data(self) -> TreeData:
        return walk(self.tp)

    def highest_s(self) -> int:
        return lib().get_highest_s(self.tp)

    def free(self):
        if self.tp:
            if self.keep is not None:
                # data belongs to numpy: drop the pointers first
                td_h = self.height
                t = self.tp.contents
                for i in range(1 << td_h):
                    t.innermost_leaves[i].contents.data.diagonal.data = None
                from .tree import node_at
                for d in range(td_h):
                    for j in range(1 << d):
                        nd = node_at(self.tp, d, j).contents
                        for c in (1, 2):
                            od = nd.children[c].leaf.contents.data.off_diagonal
                            od.u = None
                            od.v = None
            lib().free_tree_hodlr(C.byref(self.tp))
            self.tp = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def matmat_batched(trees, xs, ks, ldxs, ys, ldys, op: int = 0, precision: int = 0,
                   stream: int = 0):
    """hodlr_b200_matmat_batched_dev: Y_i = op(H_i) X_i for every tree, one
    launch per phase.  xs / ys are device addresses (ints)."""
    n = len(trees)
    arr = lambda T, v: (T * max(n, 1))(*v)
    r = lib().hodlr_b200_matmat_batched_dev(
        n, arr(C.c_void_p, [t.h for t in trees]), op, precision, arr(C.c_void_p, xs),
        arr(C.c_int, ks), arr(C.c_int, ldxs), arr(C.c_void_p, ys), arr(C.c_int, ldys),
        C.c_void_p(stream))
    if r != abi.SUCCESS:
        raise HodlrError(r, "hodlr_b200_matmat_batched_dev", lib().hodlr_b200_last_error().decode())


def batched_tuning() -> str:
    buf = C.create_string_buffer(512)
    lib().hodlr_b200_batched_tuning(buf, 512)
    return buf.value.decode()


class DeviceTree:
    """Handle of a device-resident tree (include/hmat_lib/hodlr_b200.h)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def build(cls, d_matrix_ptr: int, n: int, ld: int, height: int, tol: float,
              stream: int = 0, ms=None) -> "DeviceTree":
        out = C.c_void_p()
        ierr = C.c_int(0)
        msp = None
        if ms is not None:
            arr = (C.c_int * len(ms))(*ms)
            msp = C.cast(arr, abi.IP)
        lib().hodlr_b200_build_dev(height, n, msp, C.c_void_p(d_matrix_ptr), ld, tol, 0,
                                   C.c_void_p(stream), C.byref(out), C.byref(ierr))
        if ierr.value != abi.SUCCESS and out.value:
            # a failed build still hands over the tree it made: release it
            msg = lib().hodlr_b200_last_error().decode()
            lib().hodlr_b200_tree_free(out)
            raise HodlrError(ierr.value, "hodlr_b200_build_dev", msg)
        _check(ierr, "hodlr_b200_build_dev")
        return cls(out)

    @classmethod
    def build_batched(cls, d_matrix_ptrs, ns, lds, heights, tol: float,
                      stream: int = 0) -> list:
        """hodlr_b200_build_batched_dev: many trees in shared launches."""
        count = len(ns)
        arr = lambda T, v: (T * max(count, 1))(*v)
        out = (C.c_void_p * max(count, 1))()
        ierr = C.c_int(0)
        lib().hodlr_b200_build_batched_dev(count, arr(C.c_int, heights), arr(C.c_int, ns),
                                           arr(C.c_void_p, d_matrix_ptrs), arr(C.c_int, lds),
                                           tol, C.c_void_p(stream), out, C.byref(ierr))
        trees = [cls(C.c_void_p(out[i])) for i in range(count)] \
            if ierr.value in (abi.SUCCESS, abi.SVD_FAILURE) else []
        if ierr.value != abi.SUCCESS:
            msg = lib().hodlr_b200_last_error().decode()
            for t in trees:
                t.free()
            raise HodlrError(ierr.value, "hodlr_b200_build_batched_dev", msg)
        return trees

    @classmethod
    def build_kernel(cls, d_points_ptr: int, n: int, dim: int, kind: int, length: float,
                     diag: float, height: int, tol: float, stream: int = 0,
                     ms=None) -> "DeviceTree":
        """hodlr_b200_build_kernel_dev: the tree of a kernel matrix that is
        never formed (points column-major n x dim on the device)."""
        out = C.c_void_p()
        ierr = C.c_int(0)
        msp = None
        if ms is not None:
            arr = (C.c_int * len(ms))(*ms)
            msp = C.cast(arr, abi.IP)
        lib().hodlr_b200_build_kernel_dev(height, n, msp, C.c_void_p(d_points_ptr), dim, kind,
                                          length, diag, tol, 0, C.c_void_p(stream),
                                          C.byref(out), C.byref(ierr))
        if ierr.value != abi.SUCCESS and out.value:
            msg = lib().hodlr_b200_last_error().decode()
            lib().hodlr_b200_tree_free(out)
            raise HodlrError(ierr.value, "hodlr_b200_build_kernel_dev", msg)
        _check(ierr, "hodlr_b200_build_kernel_dev")
        return cls(out)

    @classmethod
    def of_host(cls, tree: Tree) -> "DeviceTree":
        ierr = C.c_int(0)
        h = lib().hodlr_b200_tree_from_host(tree.tp, C.byref(ierr))
        _check(ierr, "hodlr_b200_tree_from_host")
        return cls(C.c_void_p(h))

    def info(self) -> dict:
        h, n, s = C.c_int(), C.c_int(), C.c_int()
        st, ab = C.c_longlong(), C.c_longlong()
        lib().hodlr_b200_tree_info(self.h, C.byref(h), C.byref(n), C.byref(s), C.byref(st),
                                   C.byref(ab))
        return dict(height=h.value, n=n.value, max_rank=s.value, storage=st.value,
                    arena_bytes=ab.value)

    def ranks(self) -> np.ndarray:
        cnt = lib().hodlr_b200_tree_ranks(self.h, None, 0)
        buf = (C.c_int * max(cnt, 1))()
        lib().hodlr_b200_tree_ranks(self.h, buf, cnt)
        return np.array(buf[:cnt], dtype=np.int64)

    def matmat(self, d_x: int, k: int, ldx: int, d_y: int, ldy: int, op: int = 0,
               precision: int = 0, stream: int = 0):
        r = lib().hodlr_b200_matmat_dev(self.h, op, precision, C.c_void_p(d_x), k, ldx,
                                        C.c_void_p(d_y), ldy, C.c_void_p(stream))
        if r != abi.SUCCESS:
            raise HodlrError(r, "hodlr_b200_matmat_dev", lib().hodlr_b200_last_error().decode())

    def save(self, path: str):
        """hodlr_b200_tree_save."""
        r = lib().hodlr_b200_tree_save(self.h, str(path).encode())
        if r != abi.SUCCESS:
            raise HodlrError(r, "hodlr_b200_tree_save", lib().hodlr_b200_last_error().decode())

    @classmethod
    def load(cls, path: str) -> "DeviceTree":
        """hodlr_b200_tree_load."""
        out = C.c_void_p()
        r = lib().hodlr_b200_tree_load(str(path).encode(), C.byref(out))
        if r != abi.SUCCESS:
            raise HodlrError(r, "hodlr_b200_tree_load", lib().hodlr_b200_last_error().decode())
        return cls(out)

    def factorize(self, stream: int = 0) -> "Factor":
        """hodlr_b200_factorize_dev."""
        out = C.c_void_p()
        ierr = C.c_int(0)
        lib().hodlr_b200_factorize_dev(self.h, C.c_void_p(stream), C.byref(out), C.byref(ierr))
        _check(ierr, "hodlr_b200_factorize_dev")
        return Factor(out)

    def to_host(self) -> Tree:
        t = Tree(self.info()["height"])
        ierr = C.c_int(0)
        lib().hodlr_b200_tree_to_host(self.h, t.tp, C.byref(ierr))
        t.owns_data = True
        _check(ierr, "hodlr_b200_tree_to_host")
        return t

    def hxh(self, other: "DeviceTree", tol: float) -> "DeviceTree":
        out = C.c_void_p()
        ierr = C.c_int(0)
        lib().hodlr_b200_hxh_dev(self.h, other.h, tol, C.byref(out), C.byref(ierr))
        _check(ierr, "hodlr_b200_hxh_dev")
        return DeviceTree(out)

    def free(self):
        if self.h:
            lib().hodlr_b200_tree_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Factor:
    """Handle of a factorised tree (hodlr_b200_factorize_dev)."""

    def __init__(self, handle):
        self.h = handle

    def solve(self, d_b: int, k: int, ldb: int, d_x: int, ldx: int, stream: int = 0):
        r = lib().hodlr_b200_solve_dev(self.h, C.c_void_p(d_b), k, ldb, C.c_void_p(d_x), ldx,
                                       C.c_void_p(stream))
        if r != abi.SUCCESS:
            raise HodlrError(r, "hodlr_b200_solve_dev", lib().hodlr_b200_last_error().decode())

    def free(self):
        if self.h:
            lib().hodlr_b200_factor_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
