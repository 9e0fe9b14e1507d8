// HODLR x vector (one right-hand side, op N) on a device tree, the product
// behind multiply_vector (hmat_lib src/vector_algebra.c:131-197):
//   1. W_b = V_b^T x[columns of b] for every off-diagonal block of every
//      level in one launch, a warp per column of V_b;
//   2. y[leaf rows] = D x[leaf rows] + sum over levels U_b[rows] W_b in one
//      launch, a CTA per leaf and a thread per row.
// Every stored double is read once (HBM-bound); the FP64 GEMM engine would
// run its 128 x 64 tiles for a single column.  The block offsets of W are
// computed on the host once per tree and kept with it, with W itself.
#include <algorithm>

#include "dtree.h"
#include "products.h"

namespace hb {

namespace {

constexpr int kProjThreads = 256;   // 8 warps: 8 columns of V_b per CTA and pass
constexpr int kRowThreads = 128;

__global__ void __launch_bounds__(kProjThreads)
mv_project_kernel(const BlockDesc *__restrict__ blocks, const double *__restrict__ arena,
                  const double *__restrict__ x, const int *__restrict__ woff,
                  double *__restrict__ w) {
  const BlockDesc B = blocks[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int step = gridDim.y * (kProjThreads / 32);
  const double *xs = x + B.c0;
  for (int j = blockIdx.y * (kProjThreads / 32) + warp; j < B.s; j += step) {
    const double *v = arena + B.v_off + (long long)j * B.n;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int r = lane;
    for (; r + 96 < B.n; r += 128) {
      a0 = fma(v[r], xs[r], a0);
      a1 = fma(v[r + 32], xs[r + 32], a1);
      a2 = fma(v[r + 64], xs[r + 64], a2);
      a3 = fma(v[r + 96], xs[r + 96], a3);
    }
    for (; r < B.n; r += 32) a0 = fma(v[r], xs[r], a0);
    double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) w[woff[blockIdx.x] + j] = acc;
  }
}

// Four independent accumulators over c of sum_c M[c * ld] v[c].
__device__ __forceinline__ void dot4(const double *__restrict__ m, long long ld,
                                     const double *__restrict__ v, int count, double &a0,
                                     double &a1, double &a2, double &a3) {
  int c = 0;
  for (; c + 3 < count; c += 4) {
    a0 = fma(m[c * ld], v[c], a0);
    a1 = fma(m[(c + 1) * ld], v[c + 1], a1);
    a2 = fma(m[(c + 2) * ld], v[c + 2], a2);
    a3 = fma(m[(c + 3) * ld], v[c + 3], a3);
  }
  for (; c < count; ++c) a0 = fma(m[c * ld], v[c], a0);
}

__global__ void __launch_bounds__(kRowThreads)
mv_rows_kernel(const LeafDesc *__restrict__ leaves, const BlockDesc *__restrict__ blocks,
               int height, const double *__restrict__ arena, const double *__restrict__ x,
               const int *__restrict__ woff, const double *__restrict__ w,
               double *__restrict__ y) {
  const int i = blockIdx.x;
  const LeafDesc L = leaves[i];
  for (int r = threadIdx.x; r < L.m; r += blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    dot4(arena + L.off + r, L.m, x + L.r0, L.m, a0, a1, a2, a3);
    for (int d = height - 1; d >= 0; --d) {
      // the block of depth d whose rows hold leaf i: top-right if the leaf
      // lies in the first child of its depth-d ancestor, bottom-left if not
      const int j = i >> (height - d);
      const int second = (i >> (height - d - 1)) & 1;
      const BlockDesc B = blocks[2 * ((1 << d) - 1 + j) + second];
      dot4(arena + B.u_off + (L.r0 - B.r0) + r, B.m, w + woff[2 * ((1 << d) - 1 + j) + second],
           B.s, a0, a1, a2, a3);
    }
    y[L.r0 + r] = (a0 + a1) + (a2 + a3);
  }
}

}  // namespace

void matvec_f64(DeviceTree &t, const double *x, double *y, cudaStream_t s) {
  const Geometry &g = t.g;
  if (g.n == 0) return;
  const int nblocks = g.nblock();
  int max_s = 0;
  {
    std::lock_guard<std::mutex> lk(t.plan_mutex);
    if (!t.mv_woff && nblocks > 0) {
      std::vector<int> woff(nblocks);
      long long total = 0;
      for (int b = 0; b < nblocks; ++b) {
        woff[b] = (int)total;
        total += g.blocks[b].s;
      }
      HB_REQUIRE(total < (1LL << 31), INPUT_ERROR, "matvec: ranks sum past 2^31");
      HB_CUDA(cudaMalloc((void **)&t.mv_woff, sizeof(int) * nblocks));
      HB_CUDA(cudaMalloc((void **)&t.mv_w, sizeof(double) * std::max<long long>(total, 1)));
      HB_CUDA(cudaMemcpyAsync(t.mv_woff, woff.data(), sizeof(int) * nblocks,
                              cudaMemcpyHostToDevice, s));
      HB_CUDA(cudaStreamSynchronize(s));
    }
  }
  for (const BlockDesc &b : g.blocks) max_s = std::max(max_s, b.s);
  if (nblocks > 0 && max_s > 0) {
    const int gy = std::min((max_s + kProjThreads / 32 - 1) / (kProjThreads / 32), 64);
    mv_project_kernel<<<dim3(nblocks, gy), kProjThreads, 0, s>>>(t.d_blocks, t.arena, x,
                                                                t.mv_woff, t.mv_w);
    HB_LAUNCHED();
  }
  mv_rows_kernel<<<g.nleaf(), kRowThreads, 0, s>>>(t.d_leaves, t.d_blocks, g.h, t.arena, x,
                                                   t.mv_woff, t.mv_w, y);
  HB_LAUNCHED();
}

}  // namespace hb
