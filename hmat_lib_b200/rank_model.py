"""Learned rank predictor: thin wrappers over the hodlr_b200_rank_model_*
entry points (training and inference run on the GPU in the library's own
kernels) and the shipped model file.

The model maps a block's features (log2 block size, depth, ln kernel length,
five log ratios of a 16-column sketch's singular values) to log2(rank + 1)
at the build tolerance; builds with option "learned_ranks" = 1 size each
randomized sketch from it in one shot and fall back to the adaptive rule when
the a-posteriori error estimate exceeds the tolerance.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

MODEL_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rank_model.f32")
# 8 features, final rank, predicted rank, first width, fallback, final width,
# Frobenius epsilon-rank (the training target)
FEATURE_ROW = 14


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(r: int, where: str):
    if r != abi.SUCCESS:
        raise RuntimeError(f"{where}: {abi.ERROR_NAMES.get(r, r)} "
                           f"{abi.load().hodlr_b200_last_error().decode()}")


def size() -> int:
    return abi.load().hodlr_b200_rank_model_size()


def train(features: np.ndarray, targets: np.ndarray, steps: int = 3000, batch: int = 8192,
          lr: float = 3e-3, seed: int = 1):
    x = np.ascontiguousarray(features, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    p = np.zeros(size(), dtype=np.float32)
    log = np.zeros(steps // 100 + 2, dtype=np.float32)
    _check(abi.load().hodlr_b200_rank_model_train(_fp(x), _fp(t), len(t), steps, batch, lr, seed,
                                                  _fp(p), _fp(log), len(log)),
           "hodlr_b200_rank_model_train")
    return p, log[:max(1, (steps + 99) // 100)]


def predict(params: np.ndarray, features: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(features, dtype=np.float32)
    out = np.zeros(len(x), dtype=np.float32)
    _check(abi.load().hodlr_b200_rank_model_predict(_fp(p), _fp(x), len(x), _fp(out)),
           "hodlr_b200_rank_model_predict")
    return out


def gradient(params, features, targets):
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(features, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    g = np.zeros(size(), dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    _check(abi.load().hodlr_b200_rank_model_gradient(_fp(p), _fp(x), _fp(t), len(t), _fp(g),
                                                     _fp(loss)),
           "hodlr_b200_rank_model_gradient")
    return float(loss[0]), g


def adam(params, grad, m, v, step: int, lr: float):
    p = np.array(params, dtype=np.float32)
    g = np.ascontiguousarray(grad, dtype=np.float32)
    m = np.array(m, dtype=np.float32)
    v = np.array(v, dtype=np.float32)
    _check(abi.load().hodlr_b200_rank_model_adam(_fp(p), _fp(g), _fp(m), _fp(v), step, lr),
           "hodlr_b200_rank_model_adam")
    return p, m, v


def set_model(params) -> None:
    if params is None:
        _check(abi.load().hodlr_b200_rank_model_set(None, 0), "hodlr_b200_rank_model_set")
        return
    p = np.ascontiguousarray(params, dtype=np.float32)
    _check(abi.load().hodlr_b200_rank_model_set(_fp(p), len(p)), "hodlr_b200_rank_model_set")


def load_default() -> np.ndarray:
    """Reads the shipped model file and makes it the library's model."""
    p = np.fromfile(MODEL_FILE, dtype=np.float32)
    if len(p) != size():
        raise RuntimeError(f"{MODEL_FILE}: {len(p)} values, expected {size()}")
    set_model(p)
    return p


def build_features() -> np.ndarray:
    """Rows (FEATURE_ROW values) of the latest build on this thread."""
    lib = abi.load()
    rows = lib.hodlr_b200_build_features(None, 0)
    out = np.zeros((max(rows, 1), FEATURE_ROW), dtype=np.float32)
    lib.hodlr_b200_build_features(_fp(out), rows)
    return out[:rows]


def targets_of_ranks(ranks) -> np.ndarray:
    return np.log2(np.asarray(ranks, dtype=np.float64) + 1.0).astype(np.float32)
