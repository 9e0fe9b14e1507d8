"""Batched products (hodlr_b200_matmat_batched_dev): many trees of uneven
size, height, rank and column count in one launch per phase, checked
against each tree's own product through hodlr_b200_matmat_dev (FP64: same
arithmetic, summation order aside) and against the CPU oracle; graph replay
with new input values, the path without autotuning or graphs, and the
argument checks."""
import ctypes as C

import numpy as np
import pytest

from hmat_lib_b200 import abi
from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, HodlrError, batched_tuning, matmat_batched
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu

KINDS = {"gaussian": 0, "matern32": 1, "exponential": 2}


def _device_tree(n, h, kind, length, diag, seed):
    import torch
    pts = np.sort(np.random.default_rng(seed).random(n))[:, None]
    d_pts = torch.from_numpy(np.ascontiguousarray(pts)).cuda()
    a = torch.empty((n, n), dtype=torch.float64, device="cuda")
    r = abi.load().hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, 1, KINDS[kind],
                                                length, diag, C.c_void_p(a.data_ptr()), n, None)
    assert r == abi.SUCCESS
    torch.cuda.synchronize()
    return DeviceTree.build(a.data_ptr(), n, n, h, 1e-8)


@pytest.fixture(scope="module")
def batch():
    """Ten trees: sizes 256..2048, heights 1..4, three kernels."""
    rng = np.random.default_rng(5)
    trees, meta = [], []
    for i in range(10):
        n = int(rng.choice([256, 512, 1024, 2048]))
        h = int(min(4, max(1, np.log2(n // 128))))
        kind = ["exponential", "gaussian", "matern32"][i % 3]
        trees.append(_device_tree(n, h, kind, float(rng.uniform(0.05, 0.5)), 1e-2, 100 + i))
        meta.append((n, int(rng.integers(16, 129))))
    yield trees, meta
    for t in trees:
        t.free()


def _buffers(meta, op, seed):
    import torch
    rng = np.random.default_rng(seed)
    xs, ys = [], []
    for n, k in meta:
        shape = (k, n) if op == 2 else (n, k)
        xs.append(torch.from_numpy(np.asfortranarray(rng.standard_normal(shape))).cuda()
                  .t().contiguous().t())
        ys.append(torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
                  .t().contiguous().t())
    return xs, ys


def _ld(t):
    return t.stride(1)


def _single(dt, x, op, precision=0):
    import torch
    y = torch.empty_like(x)
    k = x.shape[0] if op == 2 else x.shape[1]
    dt.matmat(x.data_ptr(), k, _ld(x), y.data_ptr(), _ld(y), op=op, precision=precision)
    return y


@pytest.mark.parametrize("op", [0, 1, 2], ids=["N", "T", "L"])
def test_batched_fp64_matches_single(batch, op):
    import torch
    trees, meta = batch
    xs, ys = _buffers(meta, op, seed=op)
    ks = [x.shape[0] if op == 2 else x.shape[1] for x in xs]
    matmat_batched(trees, [x.data_ptr() for x in xs], ks, [_ld(x) for x in xs],
                   [y.data_ptr() for y in ys], [_ld(y) for y in ys], op=op)
    torch.cuda.synchronize()
    assert "phase1" in batched_tuning()
    for dt, x, y in zip(trees, xs, ys):
        want = _single(dt, x, op)
        torch.cuda.synchronize()
        assert O.rel_fro(y.cpu().numpy(), want.cpu().numpy()) < 1e-13


def test_batched_matches_oracle(batch):
    """Against the CPU oracle's product of the downloaded trees."""
    import torch
    trees, meta = batch
    xs, ys = _buffers(meta, 0, seed=11)
    matmat_batched(trees, [x.data_ptr() for x in xs], [m[1] for m in meta],
                   [_ld(x) for x in xs], [y.data_ptr() for y in ys], [_ld(y) for y in ys])
    torch.cuda.synchronize()
    for dt, x, y in list(zip(trees, xs, ys))[:4]:
        host = dt.to_host()
        want = O.multiply_dense(host.data(), x.cpu().numpy())
        assert O.rel_fro(y.cpu().numpy(), want) < 1e-12
        host.free()


def test_graph_replay_sees_new_inputs(batch):
    """Second and third calls (same signature) replay the captured graph;
    they must read the inputs' current values."""
    import torch
    trees, meta = batch
    xs, ys = _buffers(meta, 0, seed=21)
    args = ([x.data_ptr() for x in xs], [m[1] for m in meta], [_ld(x) for x in xs],
            [y.data_ptr() for y in ys], [_ld(y) for y in ys])
    launches0 = abi.load().hodlr_b200_kernel_launches()
    matmat_batched(trees, *args)
    for rep in range(2):
        for x in xs:
            x.mul_(-0.5 if rep == 0 else 3.0)
        matmat_batched(trees, *args)
    torch.cuda.synchronize()
    assert abi.load().hodlr_b200_kernel_launches() > launches0
    for dt, x, y in zip(trees, xs, ys):
        want = _single(dt, x, 0)
        torch.cuda.synchronize()
        assert O.rel_fro(y.cpu().numpy(), want.cpu().numpy()) < 1e-13


def test_without_autotune_or_graphs(batch):
    import torch
    lib = abi.load()
    trees, meta = batch
    lib.hodlr_b200_set_option(b"autotune", 0.0)
    lib.hodlr_b200_set_option(b"use_graphs", 0.0)
    try:
        xs, ys = _buffers(meta[:5], 0, seed=31)
        matmat_batched(trees[:5], [x.data_ptr() for x in xs], [m[1] for m in meta[:5]],
                       [_ld(x) for x in xs], [y.data_ptr() for y in ys], [_ld(y) for y in ys])
        torch.cuda.synchronize()
        assert " ms" not in batched_tuning()
        for dt, x, y in zip(trees[:5], xs, ys):
            want = _single(dt, x, 0)
            torch.cuda.synchronize()
            assert O.rel_fro(y.cpu().numpy(), want.cpu().numpy()) < 1e-13
    finally:
        lib.hodlr_b200_set_option(b"autotune", 1.0)
        lib.hodlr_b200_set_option(b"use_graphs", 1.0)


@pytest.mark.parametrize("shape", [0, 1, 2, 3], ids=["128x64", "64x128", "32x128", "32x256"])
def test_every_tile_shape(batch, shape):
    """Each tile shape the autotuner may pick gives the same products."""
    import torch
    lib = abi.load()
    trees, meta = batch
    lib.hodlr_b200_set_option(b"batch_shape", float(shape))
    try:
        for op in (0, 2):
            xs, ys = _buffers(meta[:6], op, seed=70 + shape)
            ks = [x.shape[0] if op == 2 else x.shape[1] for x in xs]
            matmat_batched(trees[:6], [x.data_ptr() for x in xs], ks, [_ld(x) for x in xs],
                           [y.data_ptr() for y in ys], [_ld(y) for y in ys], op=op)
            torch.cuda.synchronize()
            for dt, x, y in zip(trees[:6], xs, ys):
                want = _single(dt, x, op)
                torch.cuda.synchronize()
                assert O.rel_fro(y.cpu().numpy(), want.cpu().numpy()) < 1e-13
    finally:
        lib.hodlr_b200_set_option(b"batch_shape", -1.0)


def test_batched_mixed(batch):
    """Mixed precision: every tree once, results within the slicing error of
    each tree's FP64 product."""
    import torch
    trees, meta = batch
    xs, ys = _buffers(meta, 0, seed=41)
    for rep in range(2):
        matmat_batched(trees, [x.data_ptr() for x in xs], [m[1] for m in meta],
                       [_ld(x) for x in xs], [y.data_ptr() for y in ys], [_ld(y) for y in ys],
                       precision=1)
    torch.cuda.synchronize()
    assert abi.load().hodlr_b200_batched_check() == abi.SUCCESS
    for dt, x, y in zip(trees, xs, ys):
        want = _single(dt, x, 0)
        torch.cuda.synchronize()
        assert O.rel_fro(y.cpu().numpy(), want.cpu().numpy()) < 1e-11


def test_batched_argument_errors(batch):
    import torch
    trees, meta = batch
    xs, ys = _buffers(meta[:2], 0, seed=51)
    good = ([x.data_ptr() for x in xs], [m[1] for m in meta[:2]], [_ld(x) for x in xs],
            [y.data_ptr() for y in ys], [_ld(y) for y in ys])
    with pytest.raises(HodlrError) as e:   # the same tree twice in a mixed batch
        matmat_batched([trees[0], trees[0]], *good, precision=1)
    assert e.value.code == abi.INPUT_ERROR
    bad_ld = (good[0], good[1], [1, 1], good[3], good[4])
    with pytest.raises(HodlrError) as e:
        matmat_batched(trees[:2], *bad_ld)
    assert e.value.code == abi.INPUT_ERROR
    with pytest.raises(HodlrError) as e:   # mixed precision is op N only
        matmat_batched(trees[:2], *good, op=1, precision=1)
    assert e.value.code == abi.INPUT_ERROR
    torch.cuda.synchronize()


def test_freed_tree_invalidates_plan():
    """A plan cached for a tree that is then freed is not reused for a new
    tree, even at the same handle address."""
    import torch
    xs, ys = _buffers([(512, 32)], 0, seed=61)
    args = ([xs[0].data_ptr()], [32], [512], [ys[0].data_ptr()], [512])
    for length in (0.1, 0.4):
        dt = _device_tree(512, 2, "gaussian", length, 1.0, 7)
        matmat_batched([dt], *args)
        torch.cuda.synchronize()
        want = _single(dt, xs[0], 0)
        torch.cuda.synchronize()
        assert O.rel_fro(ys[0].cpu().numpy(), want.cpu().numpy()) < 1e-13
        dt.free()
    abi.load().hodlr_b200_batched_release()
