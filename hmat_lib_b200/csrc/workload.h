// Sub-blocks of a kernel matrix generated on the device (csrc/workload.cu).
#pragma once

#include <vector>

#include "kernelspec.cuh"

namespace hb {

struct GenBlock {
  int r0, c0;        // origin in the kernel matrix
  int rows, cols;
  double *dst;       // column-major destination
  long long ld;
};

void kernel_blocks(const KernelSpec &K, const std::vector<GenBlock> &blocks, cudaStream_t stream);

}  // namespace hb
