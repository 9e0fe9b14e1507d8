// HODLR x HODLR with recompression on the device.
#pragma once

#include "dtree.h"

namespace hb {

// out = A * B (same height and block sizes), every output off-diagonal block
// recompressed with hmat_lib's absolute truncation at `tol`.
std::shared_ptr<DeviceTree> hxh_multiply(DeviceTree &a, DeviceTree &b, double tol,
                                         cudaStream_t stream, int *status);

// Recompression of one product U V^T (U m x S, V n x S, device, column-major)
// by the routine hxh_multiply applies to every output block: QR of U and V,
// Jacobi SVD of R_U R_V^T and absolute truncation at `tol` (hmat_lib
// recompress), or with `dense` the SVD of U V^T itself (recompress_large_s).
// U' (m x r) and V' (n x r) are written contiguously (ld m, ld n) to d_uo /
// d_vo, which hold max(S, min(m, n)) columns.  Returns the Jacobi status.
int recompress_one(int m, int n, int S, const double *d_u, int ldu, const double *d_v, int ldv,
                   double tol, bool dense, double *d_uo, double *d_vo, int *rank,
                   cudaStream_t stream);

}  // namespace hb
