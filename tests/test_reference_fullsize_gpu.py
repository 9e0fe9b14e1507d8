"""Device builds and products against hmat_lib's own FP64 results at full
size (fixtures from tests/golden/make_ref_fixtures.py):

* matern2d_n32768 -- the single-tree benchmark workload (n = 32768 2D
  Matern-3/2, depth 8, tol 1e-8), built by hmat_lib patched only for 64-bit
  sizes (the unmodified constructor overflows `int` at this n);
* exp3d_n8192 -- the 3D exponential family of the n = 65536 learned-rank
  workload at a size the unmodified hmat_lib builds (depth 6, tol 1e-8).

Ranks: every block within +-1 of the reference's (LAPACK dgesdd against the
device's randomized range finder + Jacobi: a singular value within about 1%
of the threshold may fall either side).  Products: the FP64 and the
mixed-precision H X of the fixture's four seeded columns within 1e-8
relative Frobenius of the reference's multiply_hodlr_dense."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from hmat_lib_b200 import workloads as W
from hmat_lib_b200.hodlr import DeviceTree, lib as hlib
from oracle import hodlr_oracle as O

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
KINDS = {"gaussian": 0, "matern32": 1, "exponential": 2}
CASES = {
    "matern2d_n32768": dict(dim=2, seed=1, kind="matern32", length=0.1, diag=1e-2),
    "exp3d_n8192": dict(dim=3, seed=4, kind="exponential", length=0.15, diag=1e-2),
}


def _fixture(name):
    path = os.path.join(HERE, "golden", f"ref_{name}.npz")
    return np.load(path)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("matrix_free", [False, True], ids=["dense", "matrix_free"])
def test_fullsize_build_matches_reference(name, matrix_free):
    import torch
    ref = _fixture(name)
    meta = json.loads(str(ref["meta"]))
    c = CASES[name]
    n, h, tol = meta["n"], meta["height"], meta["tol"]
    lib = hlib()
    pts = W.points_morton(n, c["dim"], c["seed"])
    d_pts = torch.from_numpy(np.asfortranarray(pts).T.copy().reshape(-1)).cuda()
    kind = KINDS[c["kind"]]
    if matrix_free:
        t = DeviceTree.build_kernel(d_pts.data_ptr(), n, c["dim"], kind, c["length"], c["diag"],
                                    h, tol)
    else:
        a = torch.empty(n * n, dtype=torch.float64, device="cuda")
        assert lib.hodlr_b200_kernel_matrix_dev(C.c_void_p(d_pts.data_ptr()), n, c["dim"], kind,
                                                c["length"], c["diag"], C.c_void_p(a.data_ptr()),
                                                n, None) == 0
        t = DeviceTree.build(a.data_ptr(), n, n, h, tol)
        del a
    ranks = t.ranks()
    want = ref["ranks"].astype(np.int64)
    assert ranks.shape == want.shape
    assert int(np.abs(ranks - want).max()) <= 1, (
        f"blocks off by more than one: {int(np.sum(np.abs(ranks - want) > 1))}")
    x = W.rhs(n, meta["x_cols"], seed=meta["x_seed"])
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()          # column-major n x 4
    for precision in (0, 1):
        y = torch.zeros_like(xd)
        torch.cuda.synchronize()
        t.matmat(xd.data_ptr(), meta["x_cols"], n, y.data_ptr(), n, precision=precision)
        torch.cuda.synchronize()
        err = O.rel_fro(y.cpu().numpy().T, ref["y_ref"])
        assert err < 1e-8, (precision, err)
    t.free()
