"""ctypes mirror of the hmat_lib tree ABI and loader for libhodlr_b200.so.

The struct layouts follow include/hmat_lib/hodlr.h, which is byte-identical to
hmat_lib's include/hmat_lib/hodlr.h:7-263, so the same Python classes describe
trees produced by this library and by the reference library.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

DIAGONAL, OFFDIAGONAL, INTERNAL = 0, 1, 2

# enum ErrorCode (hmat_lib include/hmat_lib/error.h:9-16)
SUCCESS = 0
ALLOCATION_FAILURE = 1
SVD_FAILURE = 2
SVD_ALLOCATION_FAILURE = 3
INPUT_ERROR = 4
QR_FAILURE = 5
# libhodlr_b200's own status for a failed CUDA call or launch
# (include/hmat_lib/hodlr_b200.h)
HODLR_B200_CUDA_ERROR = 100

ERROR_NAMES = {
    SUCCESS: "SUCCESS",
    ALLOCATION_FAILURE: "ALLOCATION_FAILURE",
    SVD_FAILURE: "SVD_FAILURE",
    SVD_ALLOCATION_FAILURE: "SVD_ALLOCATION_FAILURE",
    INPUT_ERROR: "INPUT_ERROR",
    QR_FAILURE: "QR_FAILURE",
    HODLR_B200_CUDA_ERROR: "HODLR_B200_CUDA_ERROR",
}

DP = C.POINTER(C.c_double)
FP = C.POINTER(C.c_float)


class NodeDiagonal(C.Structure):
    _fields_ = [("data", DP), ("m", C.c_int)]


class NodeOffDiagonal(C.Structure):
    _fields_ = [("u", DP), ("v", DP), ("m", C.c_int), ("s", C.c_int), ("n", C.c_int)]


class HODLRData(C.Union):
    _fields_ = [("diagonal", NodeDiagonal), ("off_diagonal", NodeOffDiagonal)]


class HODLRInternalNode(C.Structure):
    pass


class HODLRLeafNode(C.Structure):
    _fields_ = [("type", C.c_int), ("data", HODLRData), ("parent", C.POINTER(HODLRInternalNode))]


class HODLRNode(C.Union):
    _fields_ = [("leaf", C.POINTER(HODLRLeafNode)), ("internal", C.POINTER(HODLRInternalNode))]


HODLRInternalNode._fields_ = [
    ("children", HODLRNode * 4),
    ("parent", C.POINTER(HODLRInternalNode)),
    ("m", C.c_int),
]


class TreeHODLR(C.Structure):
    _fields_ = [
        ("height", C.c_int),
        ("root", C.POINTER(HODLRInternalNode)),
        ("innermost_leaves", C.POINTER(C.POINTER(HODLRLeafNode))),
        ("len_work_queue", C.c_long),
        ("work_queue", C.POINTER(C.POINTER(HODLRInternalNode))),
        ("memory_internal_ptr", C.POINTER(HODLRInternalNode)),
        ("memory_leaf_ptr", C.POINTER(HODLRLeafNode)),
    ]


TP = C.POINTER(TreeHODLR)
IP = C.POINTER(C.c_int)
INP = C.POINTER(HODLRInternalNode)

# Signatures of the hmat_lib public API (include/hmat_lib/*.h).
HMAT_API = {
    "allocate_tree": (TP, [C.c_int, IP]),
    "allocate_tree_monolithic": (TP, [C.c_int, IP]),
    "free_tree_hodlr": (None, [C.POINTER(TP)]),
    "free_tree_data": (None, [TP]),
    "compute_construct_tree_array_sizes": (
        None, [C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
               C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "construct_tree": (
        None, [C.c_int, TP, INP, C.POINTER(HODLRLeafNode), C.POINTER(INP),
               C.POINTER(C.POINTER(HODLRLeafNode)), IP]),
    "dense_to_tree_hodlr": (C.c_int, [TP, C.c_int, IP, DP, C.c_double, IP]),
    "multiply_vector": (DP, [TP, DP, DP, IP]),
    "compute_multiply_hodlr_dense_workspace": (C.c_int, [TP, C.c_int]),
    "multiply_hodlr_dense": (DP, [TP, DP, C.c_int, C.c_int, DP, C.c_int, IP]),
    "multiply_hodlr_transpose_dense": (DP, [TP, DP, C.c_int, C.c_int, DP, C.c_int, IP]),
    "multiply_dense_hodlr": (DP, [TP, DP, C.c_int, C.c_int, DP, C.c_int, IP]),
    "multiply_internal_node_dense": (
        None, [INP, C.c_int, DP, C.c_int, C.c_int, C.POINTER(INP), DP, DP, C.c_int]),
    "multiply_internal_node_transpose_dense": (
        None, [INP, C.c_int, DP, C.c_int, C.c_int, C.POINTER(INP), DP, DP, C.c_int]),
    "multiply_dense_internal_node": (
        None, [INP, C.c_int, DP, C.c_int, C.c_int, C.POINTER(INP), DP, DP, C.c_int]),
    "multiply_hodlr_hodlr": (C.c_int, [TP, TP, TP, C.c_double, IP]),
    "get_highest_s": (C.c_int, [TP]),
}

VP = C.c_void_p

# Additive device-side API of this library (include/hmat_lib/hodlr_b200.h).
B200_API = {
    "hodlr_b200_version": (C.c_char_p, []),
    "hodlr_b200_last_error": (C.c_char_p, []),
    "hodlr_b200_build_dev": (
        C.c_int, [C.c_int, C.c_int, IP, VP, C.c_int, C.c_double, C.c_int, VP,
                  C.POINTER(VP), IP]),
    "hodlr_b200_build_batched_dev": (
        C.c_int, [C.c_int, IP, IP, C.POINTER(VP), IP, C.c_double, VP, C.POINTER(VP), IP]),
    "hodlr_b200_tree_free": (None, [VP]),
    "hodlr_b200_tree_to_host": (C.c_int, [VP, TP, IP]),
    "hodlr_b200_tree_from_host": (VP, [TP, IP]),
    "hodlr_b200_tree_info": (
        C.c_int, [VP, IP, IP, IP, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "hodlr_b200_tree_ranks": (C.c_int, [VP, IP, C.c_int]),
    "hodlr_b200_matmat_dev": (
        C.c_int, [VP, C.c_int, C.c_int, VP, C.c_int, C.c_int, VP, C.c_int, VP]),
    "hodlr_b200_hxh_dev": (C.c_int, [VP, VP, C.c_double, C.POINTER(VP), IP]),
    "hodlr_b200_recompress_dev": (C.c_int, [C.c_int, C.c_int, C.c_int, VP, C.c_int, VP, C.c_int,
                                            C.c_double, C.c_int, VP, VP, IP, VP]),
    "hodlr_b200_sync_tree": (C.c_int, [TP]),
    "hodlr_b200_kernel_launches": (C.c_longlong, []),
    "hodlr_b200_set_option": (C.c_int, [C.c_char_p, C.c_double]),
    "hodlr_b200_set_host_allocator": (None, [VP, VP]),
    "hodlr_b200_phase_times": (C.c_int, [DP, C.c_int]),
    "hodlr_b200_build_stats": (C.c_int, [DP, C.c_int]),
    "hodlr_b200_check": (C.c_int, [VP, VP]),
    "hodlr_b200_matvec_noalloc_dev": (C.c_int, [VP, VP, VP, VP]),
    "hodlr_b200_kernel_matrix_dev": (
        C.c_int, [VP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, VP, C.c_int, VP]),
    "hodlr_b200_kernel_block_dev": (
        C.c_int, [VP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                  C.c_int, C.c_int, VP, C.c_int, VP]),
    "hodlr_b200_matmat_batched_dev": (
        C.c_int, [C.c_int, C.POINTER(VP), C.c_int, C.c_int, C.POINTER(VP), IP, IP,
                  C.POINTER(VP), IP, VP]),
    "hodlr_b200_batched_tuning": (C.c_int, [C.c_char_p, C.c_int]),
    "hodlr_b200_batched_check": (C.c_int, []),
    "hodlr_b200_batched_release": (None, []),
    "hodlr_b200_rank_model_size": (C.c_int, []),
    "hodlr_b200_rank_model_set": (C.c_int, [FP, C.c_int]),
    "hodlr_b200_rank_model_get": (C.c_int, [FP, C.c_int]),
    "hodlr_b200_rank_model_train": (
        C.c_int, [FP, FP, C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong, FP, FP, C.c_int]),
    "hodlr_b200_rank_model_predict": (C.c_int, [FP, FP, C.c_int, FP]),
    "hodlr_b200_rank_model_gradient": (C.c_int, [FP, FP, FP, C.c_int, FP, FP]),
    "hodlr_b200_rank_model_adam": (C.c_int, [FP, FP, FP, FP, C.c_int, C.c_double]),
    "hodlr_b200_build_features": (C.c_int, [FP, C.c_int]),
    "hodlr_b200_build_kernel_dev": (
        C.c_int, [C.c_int, C.c_int, IP, VP, C.c_int, C.c_int, C.c_double, C.c_double,
                  C.c_double, C.c_int, VP, C.POINTER(VP), IP]),
    "hodlr_b200_factorize_dev": (C.c_int, [VP, VP, C.POINTER(VP), IP]),
    "hodlr_b200_solve_dev": (C.c_int, [VP, VP, C.c_int, C.c_int, VP, C.c_int, VP]),
    "hodlr_b200_factor_free": (None, [VP]),
    "hodlr_b200_tree_save": (C.c_int, [VP, C.c_char_p]),
    "hodlr_b200_tree_load": (C.c_int, [C.c_char_p, C.POINTER(VP)]),
}


def _declare(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libhodlr_b200.so"


def lib_path() -> str:
    return os.path.join(PACKAGE_DIR, LIB_NAME)


_LIB = None


def load(required: bool = True):
    """Load the in-tree libhodlr_b200.so (built by hmat_lib_b200.build).

    Raises if the library is missing: there is no CPU fallback for any entry
    point of this package.
    """
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        if required:
            raise RuntimeError(
                f"{LIB_NAME} not found at {path}; build it with "
                "`python -m hmat_lib_b200.build` (no CPU fallback exists)")
        return None
    lib = C.CDLL(path, mode=C.RTLD_LOCAL)
    _declare(lib, HMAT_API)
    _declare(lib, B200_API)
    _LIB = lib
    return lib


def built_source_hash(lib) -> str:
    """Digest of the sources the loaded library was built from (the last word
    of hodlr_b200_version())."""
    return lib.hodlr_b200_version().decode().rsplit(" ", 1)[-1]


def check_source_hash(lib) -> None:
    """Raises if the loaded library was not built from the sources beside
    it (rebuild with `python -m hmat_lib_b200.build`)."""
    from . import build
    want, got = build.source_hash(), built_source_hash(lib)
    if want != got:
        raise RuntimeError(f"{LIB_NAME} was built from other sources (library {got}, "
                           f"sources {want}); rebuild with `python -m hmat_lib_b200.build`")


def load_hmat_abi(path: str):
    """Load any shared library exporting the hmat_lib API (e.g. the reference
    build used as a checker) and declare its signatures."""
    lib = C.CDLL(path, mode=C.RTLD_LOCAL)
    _declare(lib, HMAT_API)
    return lib


def as_dp(a: np.ndarray):
    assert a.dtype == np.float64
    return a.ctypes.data_as(DP)


def ptr_array(ptr: DP, n: int) -> np.ndarray:
    """View (not copy) of n doubles behind a C pointer."""
    if n == 0:
        return np.zeros(0)
    return np.ctypeslib.as_array(ptr, shape=(n,))
