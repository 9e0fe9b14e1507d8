// Kernel matrices generated directly in device memory from a point set:
// A_ij = k(|p_i - p_j|) + diag * delta_ij, column-major.  Lets a caller build
// a HODLR of a kernel matrix without forming it on the host.
#include <algorithm>

#include "../../include/hmat_lib/hodlr_b200.h"
#include "kernelspec.cuh"
#include "workload.h"

namespace hb {
namespace {

// rows x cols block of the kernel matrix with origin (r0, c0); grid.y covers
// columns j0 .. j0 + gridDim.y - 1 of the block
__global__ void kernel_matrix_kernel(KernelSpec K, double *__restrict__ out, long long ld,
                                     int r0, int c0, int rows, int j0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;   // row: consecutive threads
  const int j = j0 + blockIdx.y;
  if (i >= rows) return;
  out[i + (long long)j * ld] = kernel_entry(K, r0 + i, c0 + j);
}

int launch_kernel_block(const double *d_points, int n, int dim, int kind, double length,
                        double diag, int r0, int c0, int rows, int cols, double *d_out,
                        long long ld, cudaStream_t stream) {
  KernelSpec K;
  K.pts = d_points;
  K.n = n;
  K.dim = dim;
  K.kind = kind;
  K.length = length;
  K.diag = diag;
  for (int j0 = 0; j0 < cols; j0 += 65535) {
    dim3 grid((rows + 255) / 256, std::min(65535, cols - j0));
    kernel_matrix_kernel<<<grid, 256, 0, stream>>>(K, d_out, ld, r0, c0, rows, j0);
    count_launch();
    if (cudaGetLastError() != cudaSuccess) return ALLOCATION_FAILURE;
  }
  return SUCCESS;
}

// rows x cols sub-blocks of the kernel matrix (origins r0, c0) into dense
// column-major destinations
__global__ void kernel_blocks_kernel(KernelSpec K, const GenBlock *__restrict__ blocks) {
  const GenBlock B = blocks[blockIdx.y];
  const long long total = (long long)B.rows * B.cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % B.rows), c = (int)(e / B.rows);
    B.dst[r + (long long)c * B.ld] = kernel_entry(K, B.r0 + r, B.c0 + c);
  }
}

}  // namespace
}  // namespace hb

extern "C" int hodlr_b200_kernel_matrix_dev(const double *d_points, int n, int dim, int kind,
                                            double length, double diag, double *d_out, int ld,
                                            void *stream) {
  if (!d_points || !d_out || n < 0 || dim < 1 || ld < n || kind < 0 || kind > 2)
    return INPUT_ERROR;
  if (n == 0) return SUCCESS;
  return hb::launch_kernel_block(d_points, n, dim, kind, length, diag, 0, 0, n, n, d_out, ld,
                                 (cudaStream_t)stream);
}

extern "C" int hodlr_b200_kernel_block_dev(const double *d_points, int n, int dim, int kind,
                                           double length, double diag, int r0, int c0, int rows,
                                           int cols, double *d_out, int ld, void *stream) {
  if (!d_points || !d_out || n < 0 || dim < 1 || kind < 0 || kind > 2 || r0 < 0 || c0 < 0 ||
      rows < 0 || cols < 0 || (long long)r0 + rows > n || (long long)c0 + cols > n ||
      ld < std::max(rows, 1))
    return INPUT_ERROR;
  if (rows == 0 || cols == 0) return SUCCESS;
  return hb::launch_kernel_block(d_points, n, dim, kind, length, diag, r0, c0, rows, cols, d_out,
                                 ld, (cudaStream_t)stream);
}

namespace hb {
void kernel_blocks(const KernelSpec &K, const std::vector<GenBlock> &blocks, cudaStream_t stream) {
  if (blocks.empty()) return;
  GenBlock *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(GenBlock) * blocks.size(), stream));
  HB_CUDA(cudaMemcpyAsync(d, blocks.data(), sizeof(GenBlock) * blocks.size(),
                          cudaMemcpyHostToDevice, stream));
  for (size_t off = 0; off < blocks.size(); off += 65535) {
    dim3 grid(64, (unsigned)std::min<size_t>(65535, blocks.size() - off));
    kernel_blocks_kernel<<<grid, 256, 0, stream>>>(K, d + off);
    HB_LAUNCHED();
  }
  cudaFreeAsync(d, stream);
}
}  // namespace hb
