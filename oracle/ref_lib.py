"""ctypes driver for the unmodified hmat_lib build in oracle/_ref/ --
TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline).

oracle/Makefile compiles hmat_lib's src/*.c where they lie (no copy) into
oracle/_ref/libhmat_ref.so, linked against the OpenBLAS shipped in this
image.  The library exports exactly hmat_lib's public API, whose ABI is
mirrored by hmat_lib_b200.abi, so trees it builds can be walked with
hmat_lib_b200.tree.walk.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from hmat_lib_b200 import abi
from hmat_lib_b200.tree import TreeData, walk, fill_tree, HostTreeKeepAlive

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libhmat_ref.so")

_LIB = None
_BLAS = None


def available() -> bool:
    return os.path.exists(REF_SO)


def load():
    """Load the reference build (one BLAS thread unless OPENBLAS_NUM_THREADS
    is already set: hmat_lib's OpenMP tasks and a threaded OpenBLAS do not
    mix, see hmat_lib src/constructors.c:685-699)."""
    global _LIB, _BLAS
    if _LIB is None:
        if not available():
            raise RuntimeError(f"reference build missing: {REF_SO} (run make -C oracle)")
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        _LIB = abi.load_hmat_abi(REF_SO)
        # the OpenBLAS the reference is linked to (for thread control)
        for name in os.listdir(_blas_dir()):
            if name.startswith("libopenblas"):
                _BLAS = C.CDLL(os.path.join(_blas_dir(), name), mode=C.RTLD_GLOBAL)
                break
    return _LIB


def _blas_dir():
    import sysconfig
    return os.path.join(sysconfig.get_paths()["purelib"], "opencv_python_headless.libs")


def set_blas_threads(n: int):
    load()
    if _BLAS is not None:
        _BLAS.openblas_set_num_threads(C.c_int(n))


def set_omp_threads(n: int):
    libgomp = C.CDLL("libgomp.so.1", mode=C.RTLD_GLOBAL)
    libgomp.omp_set_num_threads(C.c_int(n))


class RefTree:
    """A tree owned by the reference library."""

    def __init__(self, height: int):
        lib = load()
        ierr = C.c_int(0)
        self.tp = lib.allocate_tree_monolithic(height, C.byref(ierr))
        if ierr.value != abi.SUCCESS:
            raise RuntimeError(f"allocate_tree_monolithic: {ierr.value}")
        self.owned_data = False
        self.keep = None

    def free(self):
        if self.tp:
            lib = load()
            if self.owned_data:
                lib.free_tree_hodlr(C.byref(self.tp))
            else:
                # data points into numpy buffers: free the skeleton only
                t = self.tp.contents
                libc = C.CDLL(None)
                libc.free.argtypes = [C.c_void_p]
                for p in (t.memory_leaf_ptr, t.memory_internal_ptr, t.work_queue,
                          t.innermost_leaves):
                    libc.free(C.cast(p, C.c_void_p))
                libc.free(C.cast(self.tp, C.c_void_p))
            self.tp = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def data(self) -> TreeData:
        return walk(self.tp)


def build(a: np.ndarray, height: int, tol: float, ms=None) -> RefTree:
    """dense_to_tree_hodlr of the reference (the input is copied first since
    the reference overwrites it, src/constructors.c:576-580)."""
    lib = load()
    t = RefTree(height)
    work = np.asfortranarray(a, dtype=np.float64).copy(order="F")
    ierr = C.c_int(0)
    msp = None
    if ms is not None:
        msa = (C.c_int * len(ms))(*ms)
        msp = C.cast(msa, abi.IP)
    res = lib.dense_to_tree_hodlr(t.tp, a.shape[0], msp, abi.as_dp(work.reshape(-1, order="F")),
                                  tol, C.byref(ierr))
    if ierr.value != abi.SUCCESS or res != 0:
        raise RuntimeError(f"reference dense_to_tree_hodlr: ierr={ierr.value} info={res}")
    t.owned_data = True
    return t


def from_tree_data(td: TreeData) -> RefTree:
    t = RefTree(td.height)
    t.keep = HostTreeKeepAlive()
    fill_tree(t.tp, td, t.keep)
    return t


def multiply_dense(t: RefTree, x: np.ndarray, op: str = "N") -> np.ndarray:
    """op N: H X; T: H^T X; L: X H (X k x n)."""
    lib = load()
    xf = np.asfortranarray(x, dtype=np.float64)
    out = np.zeros_like(xf, order="F")
    ierr = C.c_int(0)
    xp = xf.ctypes.data_as(abi.DP)
    op_ = out.ctypes.data_as(abi.DP)
    if op == "N":
        lib.multiply_hodlr_dense(t.tp, xp, xf.shape[1], xf.shape[0], op_, xf.shape[0], C.byref(ierr))
    elif op == "T":
        lib.multiply_hodlr_transpose_dense(t.tp, xp, xf.shape[1], xf.shape[0], op_, xf.shape[0],
                                           C.byref(ierr))
    elif op == "L":
        lib.multiply_dense_hodlr(t.tp, xp, xf.shape[0], xf.shape[0], op_, xf.shape[0], C.byref(ierr))
    else:
        raise ValueError(op)
    if ierr.value != abi.SUCCESS:
        raise RuntimeError(f"reference multiply ({op}): ierr={ierr.value}")
    return np.asarray(out)


def multiply_vector(t: RefTree, x: np.ndarray) -> np.ndarray:
    lib = load()
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    ierr = C.c_int(0)
    lib.multiply_vector(t.tp, abi.as_dp(x), abi.as_dp(out), C.byref(ierr))
    if ierr.value != abi.SUCCESS:
        raise RuntimeError(f"reference multiply_vector: ierr={ierr.value}")
    return out


def multiply_hodlr_hodlr(t1: RefTree, t2: RefTree, tol: float) -> RefTree:
    lib = load()
    out = RefTree(t1.data().height if False else t1.tp.contents.height)
    ierr = C.c_int(0)
    res = lib.multiply_hodlr_hodlr(t1.tp, t2.tp, out.tp, tol, C.byref(ierr))
    if ierr.value != abi.SUCCESS or res != 0:
        raise RuntimeError(f"reference multiply_hodlr_hodlr: ierr={ierr.value} info={res}")
    out.owned_data = True
    return out
