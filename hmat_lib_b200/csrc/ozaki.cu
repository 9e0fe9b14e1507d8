// int8-sliced FP64 products on tcgen05 (see ozaki.h for the scheme).
//
// One CTA of 128 threads per 128 x 64 output tile.  The tile's K range is a
// list of segments, each with its own row / column scaling; K advances 64
// bytes per stage through a three-stage cp.async ring.  Thread 0 issues the
// S(S+1)/2 slice products of every 32-byte k-step into S int32 TMEM
// accumulators (group t = p + q - 2, 64 columns each) and commits each stage
// to that stage's mbarrier, which frees the buffer for the next load.  At the
// end of a segment the four warps read their 32 TMEM lanes, recombine the
// groups in FP64 and add them, scaled by 2^(e_r + f_j), to 64 FP64 registers
// per thread; the tile is written once (or added atomically for split K).
//
// Shared-memory operand layout: no swizzle, K-major, 8-row x 16-byte core
// matrices; within a 64-byte stage a row group of 8 rows holds its four
// K-chunks at 128-byte steps (leading byte offset 128) and successive row
// groups are 512 bytes apart (stride byte offset 512).
#include <algorithm>
#include <cmath>

#include "ozaki.h"
#include "umma.cuh"

namespace hb {

namespace {

constexpr int kOzThreads = 128;
constexpr int kASlice = kOzM * kOzKStage;          // bytes of one A slice per stage
constexpr int kBSlice = kOzN * kOzKStage;          // bytes of one B slice per stage
constexpr int kStageBytes = kOzSlices * (kASlice + kBSlice);
constexpr size_t kOzSmem = (size_t)kOzStages * kStageBytes;
constexpr long long kWaitTries = 1LL << 26;         // bounded barrier waits

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

__device__ __forceinline__ int core_off(int row, int chunk) {
  return (row >> 3) * 512 + chunk * 128 + (row & 7) * 16;
}

struct Cursor {
  int seg;   // absolute segment index
  int k0;    // byte offset of the stage inside the segment
};

__global__ void __launch_bounds__(kOzThreads, 1)
ozaki_gemm_kernel(const OzSeg *__restrict__ segs, const OzTile *__restrict__ tiles, double *cbase,
                  int *status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t bars[kOzStages];
  __shared__ uint32_t taddr_s;
  __shared__ int bad;

  const OzTile T = tiles[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int seg_end = T.seg0 + T.nseg;

  int nst = 0;
  for (int s = T.seg0; s < seg_end; ++s) nst += (segs[s].K + kOzKStage - 1) / kOzKStage;

  if (warp == 0) {
    umma::tmem_alloc(&taddr_s, 512);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    for (int s = 0; s < kOzStages; ++s) umma::mbar_init(&bars[s], 1);
    umma::fence_mbar_init();
    bad = 0;
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = taddr_s;

  auto settle = [&](Cursor &c) {
    while (c.seg < seg_end && c.k0 >= segs[c.seg].K) {
      ++c.seg;
      c.k0 = 0;
    }
  };
  auto advance = [&](Cursor &c) {
    c.k0 += kOzKStage;
    settle(c);
  };
  auto load_stage = [&](int buf, const Cursor &c) {
    const OzSeg G = segs[c.seg];
    uint8_t *st = sm + buf * kStageBytes;
    for (int e = tid; e < kOzSlices * kOzM * 4; e += kOzThreads) {
      const int p = e / (kOzM * 4), rem = e % (kOzM * 4), r = rem >> 2, ch = rem & 3;
      const int kb = c.k0 + ch * 16;
      const bool ok = r < T.rows && kb < G.K;
      const int8_t *src = G.a.base + p * G.a.slice_stride + (long long)r * G.a.ld + kb;
      cp_async16(st + p * kASlice + core_off(r, ch), ok ? (const void *)src : (const void *)G.a.base,
                 ok);
    }
    uint8_t *stb = st + kOzSlices * kASlice;
    for (int e = tid; e < kOzSlices * kOzN * 4; e += kOzThreads) {
      const int q = e / (kOzN * 4), rem = e % (kOzN * 4), n = rem >> 2, ch = rem & 3;
      const int kb = c.k0 + ch * 16;
      const bool ok = n < T.cols && kb < G.K;
      const int8_t *src = G.b.base + q * G.b.slice_stride + (long long)n * G.b.ld + kb;
      cp_async16(stb + q * kBSlice + core_off(n, ch), ok ? (const void *)src : (const void *)G.b.base,
                 ok);
    }
  };

  double acc[kOzN];
#pragma unroll
  for (int j = 0; j < kOzN; ++j) acc[j] = 0.0;

  Cursor ld{T.seg0, 0}, mc{T.seg0, 0};
  settle(ld);
  settle(mc);
  // prologue: two stages in flight
  for (int i = 0; i < 2; ++i) {
    if (i < nst) {
      load_stage(i % kOzStages, ld);
      advance(ld);
    }
    cp_async_commit();
  }
  constexpr uint32_t idesc = umma::idesc_s8(kOzM, kOzN);
  uint32_t inited = 0;   // accumulator groups written in the current segment (thread 0)

  for (int i = 0; i < nst; ++i) {
    const int buf = i % kOzStages;
    cp_async_wait1();
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (bad) break;
    const OzSeg G = segs[mc.seg];
    if (tid == 0) {
      const uint32_t sbase = umma::smem_u32(sm + buf * kStageBytes);
      for (int ks = 0; ks < kOzKStage / 32; ++ks) {
        if (mc.k0 + ks * 32 >= G.K) break;
#pragma unroll
        for (int p = 1; p <= kOzSlices; ++p)
#pragma unroll
          for (int q = 1; p + q <= kOzSlices + 1; ++q) {
            const int t = p + q - 2;
            const uint64_t ad =
                umma::smem_desc_noswizzle(sbase + (p - 1) * kASlice + ks * 256, 128, 512);
            const uint64_t bd = umma::smem_desc_noswizzle(
                sbase + kOzSlices * kASlice + (q - 1) * kBSlice + ks * 256, 128, 512);
            umma::mma_s8(tbase + t * kOzN, ad, bd, idesc, (inited >> t) & 1u);
            inited |= 1u << t;
          }
      }
      umma::mma_commit(&bars[buf]);
    }
    // refill the buffer last used by stage i - 1 with stage i + 2
    if (i + 2 < nst) {
      if (i >= 1) {
        const int pb = (i - 1) % kOzStages;
        if (!umma::mbar_wait_bounded(&bars[pb], ((i - 1) / kOzStages) & 1, kWaitTries)) bad = 1;
      }
      if (!bad) {
        load_stage((i + 2) % kOzStages, ld);
        advance(ld);
      }
    }
    cp_async_commit();
    // end of a segment: recombine its accumulators into the FP64 registers
    Cursor nx = mc;
    advance(nx);
    if (nx.seg != mc.seg) {
      if (!umma::mbar_wait_bounded(&bars[buf], (i / kOzStages) & 1, kWaitTries)) bad = 1;
      umma::fence_after_sync();
      const int r = tid;
      const int er = (r < T.rows) ? G.a.exp[r] : 0;
      const uint32_t lane_addr = tbase + ((uint32_t)(32 * warp) << 16);
#pragma unroll
      for (int c0 = 0; c0 < kOzN; c0 += 16) {
        double part[16];
#pragma unroll
        for (int x = 0; x < 16; ++x) part[x] = 0.0;
        // every group was written: a drained segment has at least one k-step
#pragma unroll
        for (int t = 0; t < kOzSlices; ++t) {
          int32_t v[16];
          umma::tmem_ld16(lane_addr + t * kOzN + c0, v);
          umma::tmem_ld_wait();
          const double sc = ldexp(1.0, -7 * (t + 2));
#pragma unroll
          for (int x = 0; x < 16; ++x) part[x] = fma((double)v[x], sc, part[x]);
        }
#pragma unroll
        for (int x = 0; x < 16; ++x) {
          const int j = c0 + x;
          const int fj = (j < T.cols) ? G.b.exp[j] : 0;
          acc[j] += ldexp(part[x], er + fj);
        }
      }
      umma::fence_before_sync();
      __syncthreads();
      if (tid == 0) inited = 0;
    }
    mc = nx;
  }
  cp_async_wait0();

  if (!bad && tid < T.rows) {
    const int r = tid;
#pragma unroll
    for (int j = 0; j < kOzN; ++j) {
      if (j >= T.cols) continue;
      double *c = cbase + T.c_off + r + (long long)j * T.ldc;
      if (T.atomic)
        atomicAdd(c, acc[j]);
      else
        *c = acc[j];
    }
  }
  if (bad && tid == 0) {
    atomicExch(status, 1);
    // let any MMA still in flight finish before the TMEM is released
    for (int s = 0; s < kOzStages; ++s) umma::mbar_wait_bounded(&bars[s], 0, kWaitTries);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tbase, 512);
}

// ---- slicing ---------------------------------------------------------------------

__device__ __forceinline__ int scale_exponent(double maxabs) {
  if (!(maxabs > 0.0)) return 0;
  int e;
  const double mant = frexp(maxabs, &e);   // maxabs = mant 2^e, mant in [0.5, 1)
  return mant > 127.0 / 128.0 ? e + 1 : e;
}

// exponent per row (rowwise) or per column (colwise) of the source
__global__ void slice_exp_kernel(const SliceJob *__restrict__ jobs) {
  const SliceJob J = jobs[blockIdx.y];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int count = J.rowwise ? J.m : J.k;
  for (int v = blockIdx.x * nw + warp; v < count; v += gridDim.x * nw) {
    double mx = 0.0;
    if (J.rowwise) {
      for (int c = lane; c < J.k; c += 32) mx = fmax(mx, fabs(J.src[v + (long long)c * J.ld]));
    } else {
      const double *col = J.src + (long long)v * J.ld;
      for (int r = lane; r < J.m; r += 32) mx = fmax(mx, fabs(col[r]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) J.exp[v] = scale_exponent(mx);
  }
}

// 16 consecutive K positions of one row (rowwise) or column (colwise) per
// thread; every slice gets one aligned 16-byte store; padding is zero.
__global__ void slice_kernel(const SliceJob *__restrict__ jobs) {
  const SliceJob J = jobs[blockIdx.y];
  const int lines = J.rowwise ? J.m : J.k;       // rows of the sliced operand
  const int chunks = J.dld / 16;                 // 16-byte chunks per line (padded)
  const long long total = (long long)lines * chunks;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int line = (int)(e % lines), ch = (int)(e / lines);
    const int ex = J.exp[line];
    int8_t out[kOzSlices][16];
#pragma unroll
    for (int x = 0; x < 16; ++x) {
      const int kk = ch * 16 + x;
      double y = 0.0;
      if (J.rowwise) {
        if (kk < J.k) y = J.src[line + (long long)kk * J.ld];
      } else {
        if (kk < J.m) y = J.src[kk + (long long)line * J.ld];
      }
      y = ldexp(y, -ex);
#pragma unroll
      for (int p = 0; p < kOzSlices; ++p) {
        y *= 128.0;
        const double a = rint(y);
        out[p][x] = (int8_t)a;
        y -= a;
      }
    }
#pragma unroll
    for (int p = 0; p < kOzSlices; ++p) {
      int4 w;
      memcpy(&w, out[p], 16);
      *reinterpret_cast<int4 *>(J.dst + p * J.slice_stride + (long long)line * J.dld + ch * 16) = w;
    }
  }
}

}  // namespace

void ozaki_gemm(const OzSeg *d_segs, const OzTile *d_tiles, int ntiles, double *cbase,
                int *d_status, cudaStream_t stream) {
  if (ntiles <= 0) return;
  static bool configured = false;
  if (!configured) {
    HB_CUDA(cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kOzSmem));
    configured = true;
  }
  for (int off = 0; off < ntiles; off += 65535) {
    const int cnt = std::min(65535, ntiles - off);
    ozaki_gemm_kernel<<<cnt, kOzThreads, kOzSmem, stream>>>(d_segs, d_tiles + off, cbase,
                                                             d_status);
    HB_LAUNCHED();
  }
}

void ozaki_slice(const std::vector<SliceJob> &jobs, cudaStream_t stream) {
  if (jobs.empty()) return;
  SliceJob *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(SliceJob) * jobs.size(), stream));
  HB_CUDA(cudaMemcpyAsync(d, jobs.data(), sizeof(SliceJob) * jobs.size(), cudaMemcpyHostToDevice,
                          stream));
  for (size_t off = 0; off < jobs.size(); off += 65535) {
    dim3 grid(16, (unsigned)std::min<size_t>(65535, jobs.size() - off));
    slice_exp_kernel<<<grid, 256, 0, stream>>>(d + off);
    HB_LAUNCHED();
    slice_kernel<<<grid, 256, 0, stream>>>(d + off);
    HB_LAUNCHED();
  }
  cudaFreeAsync(d, stream);
}

}  // namespace hb
