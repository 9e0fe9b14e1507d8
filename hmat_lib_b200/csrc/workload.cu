// Kernel matrices generated directly in device memory from a point set:
// A_ij = k(|p_i - p_j|) + diag * delta_ij, column-major.  Lets a caller build
// a HODLR of a kernel matrix without forming it on the host.
#include "../../include/hmat_lib/hodlr_b200.h"
#include "common.h"

namespace hb {
namespace {

__global__ void kernel_matrix_kernel(const double *__restrict__ pts, int n, int dim, int kind,
                                     double length, double diag, double *__restrict__ out,
                                     long long ld, int j0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;   // row: consecutive threads
  const int j = j0 + blockIdx.y;
  if (i >= n) return;
  double r2 = 0.0;
  for (int a = 0; a < dim; ++a) {
    const double d = pts[i + (long long)a * n] - pts[j + (long long)a * n];
    r2 = fma(d, d, r2);
  }
  const double r = sqrt(r2);
  double v;
  if (kind == 0) {
    v = exp(-r2 / (2.0 * length * length));           // Gaussian
  } else if (kind == 1) {
    const double t = 1.7320508075688772 * r / length;  // Matern-3/2
    v = (1.0 + t) * exp(-t);
  } else {
    v = exp(-r / length);                              // exponential
  }
  if (i == j) v += diag;
  out[i + (long long)j * ld] = v;
}

}  // namespace
}  // namespace hb

extern "C" int hodlr_b200_kernel_matrix_dev(const double *d_points, int n, int dim, int kind,
                                            double length, double diag, double *d_out, int ld,
                                            void *stream) {
  if (!d_points || !d_out || n < 0 || dim < 1 || ld < n || kind < 0 || kind > 2)
    return INPUT_ERROR;
  if (n == 0) return SUCCESS;
  for (int j0 = 0; j0 < n; j0 += 65535) {
    dim3 grid((n + 255) / 256, std::min(65535, n - j0));
    hb::kernel_matrix_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
        d_points, n, dim, kind, length, diag, d_out, ld, j0);
    hb::count_launch();
    if (cudaGetLastError() != cudaSuccess) return ALLOCATION_FAILURE;
  }
  return SUCCESS;
}
