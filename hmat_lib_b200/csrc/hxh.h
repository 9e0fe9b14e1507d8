// HODLR x HODLR with recompression on the device.
#pragma once

#include "dtree.h"

namespace hb {

// out = A * B (same height and block sizes), every output off-diagonal block
// recompressed with hmat_lib's absolute truncation at `tol`.
std::shared_ptr<DeviceTree> hxh_multiply(DeviceTree &a, DeviceTree &b, double tol,
                                         cudaStream_t stream, int *status);

}  // namespace hb
