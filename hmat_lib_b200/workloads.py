"""Seeded synthetic workloads: point sets, kernel matrices, right-hand sides.

These reproduce the shapes and value distributions of the benchmark
configurations (kernel matrices on sorted / Morton-ordered random points)
and the small matrices hmat_lib's unit tests use
(hmat_lib tests/utils/common_data.c).  All matrices are FP64; functions
return numpy arrays in column-major (Fortran) order where a matrix is
returned.
"""
from __future__ import annotations

import numpy as np


# ------------------------------------------------------------ points ---

def _spread_bits(v: np.ndarray, bits: int, stride: int) -> np.ndarray:
    v = v.astype(np.uint64)
    out = np.zeros_like(v)
    for b in range(bits):
        out |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(stride * b)
    return out


def morton_order(points: np.ndarray, bits: int = 21) -> np.ndarray:
    """Permutation sorting points of [0,1]^d (d = 2 or 3) along the Z-order
    curve: each coordinate quantised to `bits` bits, bits interleaved
    (x lowest)."""
    d = points.shape[1]
    q = np.clip((points * (1 << bits)).astype(np.int64), 0, (1 << bits) - 1)
    code = np.zeros(points.shape[0], dtype=np.uint64)
    for a in range(d):
        code |= _spread_bits(q[:, a], bits, d) << np.uint64(a)
    return np.argsort(code, kind="stable")


def points_1d_sorted(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.random(n))[:, None]


def points_morton(n: int, dim: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = rng.random((n, dim))
    return p[morton_order(p)]


# ----------------------------------------------------------- kernels ---

KERNELS = ("gaussian", "matern32", "exponential")


def kernel_values(kind: str, r: np.ndarray, length: float) -> np.ndarray:
    if kind == "gaussian":
        return np.exp(-(r * r) / (2.0 * length * length))
    if kind == "matern32":
        t = np.sqrt(3.0) * r / length
        return (1.0 + t) * np.exp(-t)
    if kind == "exponential":
        return np.exp(-r / length)
    raise ValueError(kind)


def kernel_matrix(points: np.ndarray, kind: str, length: float, diag: float) -> np.ndarray:
    """A_ij = k(|p_i - p_j|) + diag * delta_ij (column-major, host)."""
    diff = points[:, None, :] - points[None, :, :]
    r = np.sqrt(np.sum(diff * diff, axis=-1))
    a = kernel_values(kind, r, length)
    a[np.diag_indices_from(a)] += diag
    return np.asfortranarray(a)


def kernel_matrix_blocked(points: np.ndarray, kind: str, length: float, diag: float,
                          cols: int = 512) -> np.ndarray:
    """kernel_matrix built a block of columns at a time (column-major), so
    large n needs no n x n x dim temporaries."""
    n = points.shape[0]
    a = np.empty((n, n), order="F")
    for j0 in range(0, n, cols):
        j1 = min(n, j0 + cols)
        d = points[:, None, :] - points[None, j0:j1, :]
        a[:, j0:j1] = kernel_values(kind, np.sqrt(np.einsum("ijk,ijk->ij", d, d)), length)
    a[np.arange(n), np.arange(n)] += diag
    return a


# ------------------------------------------------- benchmark workloads ---

# The five workload shapes: (points, kernel, length, diagonal shift,
# height, tolerance, right-hand sides).
WORKLOADS = {
    "gauss1d_n1024": dict(n=1024, dim=1, seed=0, kind="gaussian", length=0.2, diag=1.0,
                          height=3, tol=1e-10, k=1),
    "matern2d_n32768": dict(n=32768, dim=2, seed=1, kind="matern32", length=0.1, diag=1e-2,
                            height=8, tol=1e-8, k=256),
    "exp3d_n65536": dict(n=65536, dim=3, seed=4, kind="exponential", length=0.15, diag=1e-2,
                         height=9, tol=1e-8, k=128),
}


def workload_points(name: str, n: int | None = None) -> np.ndarray:
    w = WORKLOADS[name]
    n = w["n"] if n is None else n
    if w["dim"] == 1:
        return points_1d_sorted(n, w["seed"])
    return points_morton(n, w["dim"], w["seed"])


def rhs(n: int, k: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed + 1000)
    return np.asfortranarray(rng.standard_normal((n, k)))


def uneven_batch(count: int = 512, seed: int = 2):
    """The uneven batch: sizes from {1024, 2048, 4096, 8192}, exponential
    kernels with l ~ U[0.05, 0.5] on sorted 1D points, 16-128 right-hand
    sides each (leaf 128, tol 1e-8)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice([1024, 2048, 4096, 8192]))
        length = float(rng.uniform(0.05, 0.5))
        k = int(rng.integers(16, 129))
        pts = np.sort(rng.random(n))[:, None]
        out.append(dict(n=n, length=length, k=k, points=pts,
                        height=int(np.log2(n // 128)), tol=1e-8))
    return out


def hxh_pair(n: int = 16384, seed: int = 3):
    """Points and kernel choices of the HODLR x HODLR workload: A from a
    Gaussian kernel (l = 0.1), B from Matern-3/2 (l = 0.2), both + 1.0 I on
    the same sorted 1D points."""
    pts = points_1d_sorted(n, seed)
    return pts, ("gaussian", 0.1, 1.0), ("matern32", 0.2, 1.0)


# --------------------------------------- matrices of hmat_lib's tests ---

def laplacian(m: int) -> np.ndarray:
    """Tridiagonal 2 / -1 (hmat_lib tests/utils/common_data.c:27-41)."""
    a = 2.0 * np.eye(m) - np.eye(m, k=1) - np.eye(m, k=-1)
    return np.asfortranarray(a)


def laplacian_converse(m: int) -> np.ndarray:
    """Tridiagonal -1 / 2 (hmat_lib tests/utils/common_data.c:44-56)."""
    a = -1.0 * np.eye(m) + 2.0 * (np.eye(m, k=1) + np.eye(m, k=-1))
    return np.asfortranarray(a)


def laplacian_corners(m: int, symmetric: bool) -> np.ndarray:
    """Laplacian with 0.5 written at column-major flat index m-1 (the
    bottom-left corner) and, if symmetric, at m*(m-1) (top-right)."""
    a = laplacian(m)
    a[m - 1, 0] = 0.5
    if symmetric:
        a[0, m - 1] = 0.5
    return a


def decay_matrix(vec: np.ndarray, scale: float) -> np.ndarray:
    """exp(-scale |v_i - v_j|) (hmat_lib tests/utils/common_data.c:114-126)."""
    return np.asfortranarray(np.exp(-scale * np.abs(vec[:, None] - vec[None, :])))
