// HODLR x vector on a device-resident tree without allocating any memory.
//
// Some callers cannot allocate device memory while they run: an iterative
// solver whose memory pool already holds (nearly) all of HBM, or
// latency-critical code that cannot afford the implicit device
// synchronisation of cudaMalloc / cudaFree.  For them the product's only
// scratch -- the projections W_b = V_b^T x of every off-diagonal block -- lives
// in a fixed array of device memory inside this file instead of a per-call
// allocation.  The caller passes the tree, x and y; nothing is allocated on
// the host or the device.
//
// Limits: sum over blocks of the ranks <= kNoAllocW (65536) and at most
// kNoAllocBlocks (4096) off-diagonal blocks (height <= 11).  The array takes
// 528 KiB on every GPU that loads the library, until the process exits.
// Every call shares it and leaves its contents behind; all of it is rewritten
// before it is read, so nothing needs clearing, but calls that overlap on the
// GPU (different streams, no ordering) race on it.
#include <mutex>

#include "../../include/hmat_lib/hodlr_b200.h"
#include "dtree.h"

namespace hb {
namespace {

constexpr int kNoAllocW = 65536;          // doubles of projections
constexpr int kNoAllocBlocks = 4096;      // int offsets, one per block
constexpr int kNoAllocDoubles = kNoAllocW + kNoAllocBlocks / 2;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// Host-side device addresses of g_noalloc_scratch, one per device.  The
// symbol's name in host code is only a host-side stand-in, so the address
// must come from cudaGetSymbolAddress with the device current.
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// W offset of every block: exclusive prefix sum of the ranks, by one CTA of
// 1024 threads (four blocks per thread, warp scans, then a scan of the warp
// totals).  nblocks <= kNoAllocBlocks = 4096.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads)
noalloc_offsets_kernel(const BlockDesc *__restrict__ blocks, int nblocks, int *__restrict__ woff) {
  __shared__ int warp_total[kScanThreads / 32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  int v[4], local = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int b = 4 * t + q;
    v[q] = b < nblocks ? blocks[b].s : 0;
    local += v[q];
  }
  int incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_total[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int w = warp_total[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_total[lane] = w;                 // inclusive totals of warps 0..lane
  }
  __syncthreads();
  int acc = incl - local + (wid > 0 ? warp_total[wid - 1] : 0);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int b = 4 * t + q;
    if (b < nblocks) woff[b] = acc;
    acc += v[q];
  }
}

// W_b[j] = V_b[:, j] . x[c0 : c0 + n], one warp per column j.
__global__ void noalloc_project_kernel(const BlockDesc *__restrict__ blocks,
                                       const double *__restrict__ arena,
                                       const double *__restrict__ x,
                                       const int *__restrict__ woff, double *__restrict__ w) {
  const BlockDesc B = blocks[blockIdx.x];
  const int lane = threadIdx.x & 31;
  const int j = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= B.s) return;
  const double *v = arena + B.v_off + (long long)j * B.n;
  const double *xs = x + B.c0;
  double acc = 0.0;
  for (int r = lane; r < B.n; r += 32) acc = fma(v[r], xs[r], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) w[woff[blockIdx.x] + j] = acc;
}

// y[leaf rows] = D x[leaf rows] + sum over levels of U_b[rows] W_b, one CTA
// per leaf, one thread per row.
__global__ void noalloc_rows_kernel(const LeafDesc *__restrict__ leaves,
                                    const BlockDesc *__restrict__ blocks, int height,
                                    const double *__restrict__ arena,
                                    const double *__restrict__ x, const int *__restrict__ woff,
                                    const double *__restrict__ w, int any_rank,
                                    double *__restrict__ y) {
  const int i = blockIdx.x;
  const LeafDesc L = leaves[i];
  const double *D = arena + L.off;
  for (int r = threadIdx.x; r < L.m; r += blockDim.x) {
    double acc = 0.0;
    for (int c = 0; c < L.m; ++c) acc = fma(D[r + (long long)c * L.m], x[L.r0 + c], acc);
    for (int d = any_rank ? height - 1 : -1; d >= 0; --d) {
      const int j = i >> (height - d);
      const bool top = ((i >> (height - d - 1)) & 1) == 0;
      const int b = 2 * ((1 << d) - 1 + j) + (top ? 0 : 1);
      const BlockDesc B = blocks[b];
      const double *u = arena + B.u_off + (L.r0 - B.r0) + r;
      const double *wb = w + woff[b];
      for (int c = 0; c < B.s; ++c) acc = fma(u[(long long)c * B.m], wb[c], acc);
    }
    y[L.r0 + r] = acc;
  }
}

// Address of the scratch array on device `dev`, which must be the current
// device: the first call on a device looks it up (and must therefore come
// before any stream capture).
double *scratch_for_device(int dev) {
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_scratch_mutex);
  if (g_scratch_addr[dev] == nullptr) {
    double *ptr = nullptr;
    if (cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch) != cudaSuccess) {
      (void)cudaGetLastError();
      return nullptr;
    }
    g_scratch_addr[dev] = ptr;
  }
  return g_scratch_addr[dev];
}

// After a launch: a configuration error is this call's failure.
bool launch_failed() {
  count_launch();
  return cudaGetLastError() != cudaSuccess;
}

int launch_error() {
  set_last_error_static("hodlr_b200_matvec_noalloc_dev: kernel launch failed");
  return HODLR_B200_CUDA_ERROR;
}

}  // namespace
}  // namespace hb

extern "C" int hodlr_b200_matvec_noalloc_dev(hodlr_b200_tree t, const double *d_x, double *d_y,
                                             void *stream) {
  using namespace hb;
  if (!t || !t->p || !d_x || !d_y) return INPUT_ERROR;
  // A CUDA error left behind by earlier asynchronous work (cudaGetLastError
  // also clears it) is reported as such rather than as a failure of this call.
  if (cudaGetLastError() != cudaSuccess) {
    set_last_error_static(
        "hodlr_b200_matvec_noalloc_dev: a CUDA error from earlier work was pending (now "
        "cleared); nothing was launched");
    return HODLR_B200_CUDA_ERROR;
  }
  const DeviceTree &T = *t->p;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != T.device) {
    (void)cudaGetLastError();
    set_last_error_static(
        "hodlr_b200_matvec_noalloc_dev: the current device is not the device that holds the "
        "tree; make it current (cudaSetDevice) before the call");
    return INPUT_ERROR;
  }
  const Geometry &g = T.g;
  const int nblocks = g.nblock();
  long long total = 0;
  int max_s = 0;
  for (const BlockDesc &b : g.blocks) {
    total += b.s;
    max_s = b.s > max_s ? b.s : max_s;
  }
  if (total > kNoAllocW || nblocks > kNoAllocBlocks) {
    set_last_error_static(
        "hodlr_b200_matvec_noalloc_dev: the tree's ranks sum to more than 65536 or it has more "
        "than 4096 off-diagonal blocks, the capacity of the fixed device scratch");
    return INPUT_ERROR;
  }
  if (g.n == 0) return SUCCESS;
  double *scratch = scratch_for_device(dev);
  if (scratch == nullptr) {
    set_last_error_static(
        "hodlr_b200_matvec_noalloc_dev: cudaGetSymbolAddress of the fixed scratch failed");
    return HODLR_B200_CUDA_ERROR;
  }
  double *w = scratch;
  int *woff = reinterpret_cast<int *>(scratch + kNoAllocW);
  cudaStream_t s = (cudaStream_t)stream;
  if (max_s > 0) {
    noalloc_offsets_kernel<<<1, kScanThreads, 0, s>>>(T.d_blocks, nblocks, woff);
    if (launch_failed()) return launch_error();
    {
      dim3 grid(nblocks, (max_s + 7) / 8);
      noalloc_project_kernel<<<grid, 256, 0, s>>>(T.d_blocks, T.arena, d_x, woff, w);
      if (launch_failed()) return launch_error();
    }
  }
  {
    // one thread per leaf row: as many threads as the largest leaf has rows
    // (rounded to whole warps, at most 256; longer leaves loop)
    int max_m = 1;
    for (int m : g.leaf_m) max_m = m > max_m ? m : max_m;
    const int threads = max_m >= 256 ? 256 : (max_m + 31) / 32 * 32;
    noalloc_rows_kernel<<<g.nleaf(), threads, 0, s>>>(T.d_leaves, T.d_blocks, g.h, T.arena, d_x,
                                                      woff, w, max_s > 0 ? 1 : 0, d_y);
    if (launch_failed()) return launch_error();
  }
  return SUCCESS;
}
