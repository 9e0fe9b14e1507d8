// int8-sliced FP64 products on tcgen05 (see ozaki.h for the scheme and the
// blocked operand layout).
//
// Persistent kernel, one CTA of six warps per SM, tiles taken round-robin:
//   warp 0 (one thread)  producer: per K-block one bulk copy of the A block
//                        (all S slices of 128 lines) and one of the B block
//                        into a six-stage ring, completion on full[stage];
//   warp 1 (one thread)  MMA issuer: per K-block the S(S+1)/2 slice products
//                        as 8 MMAs (slice p of A against slices q = 1 .. S+1-p
//                        of B, which sit next to each other in shared memory,
//                        so one MMA of N = (S+1-p) nw covers accumulator groups
//                        t = p + q - 2 stored side by side in TMEM), commit to
//                        empty[stage]; after the tile's last K-block a commit
//                        to tmem_full;
//   warps 2-5            epilogue: wait tmem_full, read the S int32 groups of
//                        their 32 TMEM lanes, recombine in FP64, scale by
//                        2^(e_r + f_j), release the accumulators (tmem_empty),
//                        store or atomically add the tile.
// The warp also owns the TMEM allocation (512 columns: S groups of <= 64).
// Every barrier wait is bounded; a wait that runs out sets the CTA's abort
// flag, every role leaves its loop, the producer waits (bounded) for its
// copies in flight, the MMA thread for its MMAs, and the kernel reports
// status 1 and returns.
#include <algorithm>
#include <cmath>

#include "ozaki.h"
#include "umma.cuh"

namespace hb {

namespace {

constexpr int kThreads = 192;
constexpr int kStages = 6;
constexpr int kStageBytes = kOzABlock + oz_bblock(kOzMaxNw);   // 36864
constexpr size_t kSmem = (size_t)kStages * kStageBytes;        // 221184
constexpr long long kWaitTries = 1LL << 26;
constexpr int kSliceBytesA = kOzRowsA * kOzKBlock;              // 4096: one slice of an A block

// Bounded wait that also gives up when another role has aborted.
__device__ __forceinline__ bool wait_or_abort(uint64_t *bar, uint32_t parity, volatile int *bad) {
  for (long long i = 0; i < kWaitTries; ++i) {
    if (umma::mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && *bad) return false;
  }
  return false;
}

__global__ void __launch_bounds__(kThreads, 1)
ozaki_gemm_kernel(const OzSeg *__restrict__ segs, const OzTile *__restrict__ tiles, int ntiles,
                  double *cbase, int *status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(8) uint64_t empty[kStages];
  __shared__ __align__(8) uint64_t tmem_full, tmem_empty, mma_done;
  __shared__ uint32_t taddr_s;
  __shared__ volatile int bad;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 1) {
    umma::tmem_alloc(&taddr_s, 512);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    umma::mbar_init(&tmem_full, 1);
    umma::mbar_init(&tmem_empty, 4);
    umma::mbar_init(&mma_done, 1);
    umma::fence_mbar_init();
    bad = 0;
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = taddr_s;

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      long long g = 0;   // K-blocks issued by this CTA
      for (int tile = blockIdx.x; tile < ntiles && !bad; tile += gridDim.x) {
        const OzTile T = tiles[tile];
        const uint32_t bbytes = (uint32_t)oz_bblock(T.nw);
        for (int s = T.seg0; s < T.seg0 + T.nseg && !bad; ++s) {
          const OzSeg G = segs[s];
          for (int kb = 0; kb < G.nkb; ++kb) {
            const int st = (int)(g % kStages);
            const long long use = g / kStages;
            if (use > 0 && !wait_or_abort(&empty[st], (uint32_t)((use - 1) & 1), &bad)) {
              bad = 1;
              break;
            }
            uint8_t *dst = sm + st * kStageBytes;
            umma::mbar_expect_tx(&full[st], (uint32_t)kOzABlock + bbytes);
            umma::bulk_g2s(dst, G.a + (long long)kb * kOzABlock, kOzABlock, &full[st]);
            umma::bulk_g2s(dst + kOzABlock, G.b + (long long)kb * bbytes, bbytes, &full[st]);
            ++g;
          }
        }
      }
      // copies still in flight land before the CTA may exit
      for (long long q = std::max(0LL, g - kStages); q < g; ++q)
        umma::mbar_wait_bounded(&full[q % kStages], (uint32_t)((q / kStages) & 1), kWaitTries);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      long long g = 0;
      int lt = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < ntiles && ok && !bad; tile += gridDim.x, ++lt) {
        const OzTile T = tiles[tile];
        if (lt > 0 && !wait_or_abort(&tmem_empty, (uint32_t)((lt - 1) & 1), &bad)) {
          ok = false;
          break;
        }
        umma::fence_after_sync();
        const int nw = T.nw;
        const int maxcnt = min(kOzSlices, 256 / nw);
        const uint32_t bslice = (uint32_t)nw * kOzKBlock;
        bool first = true;
        for (int s = T.seg0; s < T.seg0 + T.nseg && ok; ++s) {
          const int nkb = segs[s].nkb;
          for (int kb = 0; kb < nkb; ++kb, ++g) {
            const int st = (int)(g % kStages);
            if (!wait_or_abort(&full[st], (uint32_t)((g / kStages) & 1), &bad)) {
              ok = false;
              break;
            }
            umma::fence_after_sync();
            const uint32_t sa = umma::smem_u32(sm + st * kStageBytes);
            const uint32_t sb = sa + kOzABlock;
#pragma unroll
            for (int p = 1; p <= kOzSlices; ++p) {
              const uint64_t ad = umma::smem_desc_noswizzle(sa + (p - 1) * kSliceBytesA, 128, 256);
              for (int q0 = 1; q0 <= kOzSlices + 1 - p;) {
                const int cnt = min(kOzSlices + 2 - p - q0, maxcnt);
                const uint64_t bd = umma::smem_desc_noswizzle(sb + (q0 - 1) * bslice, 128, 256);
                umma::mma_s8(tbase + (uint32_t)((p + q0 - 2) * nw), ad, bd,
                             umma::idesc_s8(kOzRowsA, cnt * nw), (first && p == 1) ? 0u : 1u);
                q0 += cnt;
              }
            }
            first = false;
            umma::mma_commit(&empty[st]);
          }
        }
        if (ok) umma::mma_commit(&tmem_full);
      }
      if (!ok) bad = 1;
      // every MMA issued so far completes before the accumulators are freed
      umma::mma_commit(&mma_done);
      umma::mbar_wait_bounded(&mma_done, 0, kWaitTries);
    }
  } else {
    // ---------------- epilogue ----------------
    const int quarter = warp & 3;   // TMEM lanes 32 quarter .. 32 quarter + 31
    const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
    const int r = 32 * quarter + lane;
    int lt = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++lt) {
      if (__any_sync(0xffffffffu, bad)) break;
      const OzTile T = tiles[tile];
      const bool ready = wait_or_abort(&tmem_full, (uint32_t)(lt & 1), &bad);
      if (!__all_sync(0xffffffffu, ready)) {
        bad = 1;
        break;
      }
      umma::fence_after_sync();
      const int nw = T.nw;
      const bool row_ok = r < T.rows;
      const int er = row_ok ? T.rexp[r] : 0;
      double *crow = cbase + T.c_off + r;
      for (int c0 = 0; c0 < nw; c0 += 16) {
        int32_t v[kOzSlices][16];
#pragma unroll
        for (int t = 0; t < kOzSlices; ++t) umma::tmem_ld16(lane_addr + t * nw + c0, v[t]);
        umma::tmem_ld_wait();
        if (row_ok) {
#pragma unroll
          for (int x = 0; x < 16; ++x) {
            const int j = c0 + x;
            if (j >= T.cols) break;
            // sum_t v_t 2^(-7 t), then the common factor 2^(e_r + f_j - 14)
            double acc = (double)v[kOzSlices - 1][x];
#pragma unroll
            for (int t = kOzSlices - 2; t >= 0; --t) acc = fma(acc, 0x1p-7, (double)v[t][x]);
            const double val = ldexp(acc, er + T.cexp[j] - 14);
            double *c = crow + (long long)j * T.ldc;
            if (T.atomic)
              atomicAdd(c, val);
            else
              *c = val;
          }
        }
      }
      umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(&tmem_empty);
    }
  }

  __syncwarp();
  umma::fence_before_sync();
  __syncthreads();
  if (bad && tid == 0) atomicExch(status, 1);
  if (warp == 1) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tbase, 512);
  }
}

// ---- exponents and slicing ---------------------------------------------------------

__device__ __forceinline__ int scale_exponent(unsigned long long bits) {
  const double maxabs = __longlong_as_double((long long)bits);
  if (!(maxabs > 0.0)) return 0;
  int e;
  const double mant = frexp(maxabs, &e);   // maxabs = mant 2^e, mant in [0.5, 1)
  return mant > 127.0 / 128.0 ? e + 1 : e;
}

template <class Job>
__device__ __forceinline__ int find_job(const Job *jobs, int njobs, long long item) {
  int lo = 0, hi = njobs - 1;   // last job with item0 <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].item0 <= item)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Work items are warps: a line (K contiguous: lanes split K) or 32 lines (one
// per lane, loop over K).
__global__ void max_kernel(const MaxJob *__restrict__ jobs, int njobs, long long items,
                           const double *xbase) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long it = w0; it < items; it += nw) {
    const MaxJob &J = jobs[find_job(jobs, njobs, it)];
    const double *src = J.src ? J.src : xbase;
    const long long local = it - J.item0;
    if (J.s_k == 1) {
      const double *row = src + local * J.s_line;
      double mx = 0.0;
      for (int k = lane; k < J.K; k += 32) mx = fmax(mx, fabs(row[k]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0 && mx > 0.0)
        atomicMax(J.out + local, (unsigned long long)__double_as_longlong(mx));
    } else {
      const long long line = local * 32 + lane;
      if (line < J.lines) {
        double mx = 0.0;
        const double *p = src + line * J.s_line;
        for (int k = 0; k < J.K; ++k) mx = fmax(mx, fabs(p[(long long)k * J.s_k]));
        if (mx > 0.0) atomicMax(J.out + line, (unsigned long long)__double_as_longlong(mx));
      }
    }
  }
}

// One item = 16 consecutive K positions of one line: six aligned 16-byte
// stores, one per slice.  Lines vary fastest, so eight neighbouring items
// fill one 128-byte core matrix.
__global__ void slice_kernel(const SliceJob *__restrict__ jobs, int njobs, long long items,
                             const double *xbase) {
  for (long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x; it < items;
       it += (long long)gridDim.x * blockDim.x) {
    const SliceJob &J = jobs[find_job(jobs, njobs, it)];
    const double *src = J.src ? J.src : xbase;
    const long long local = it - J.item0;
    const int L = J.ntiles * J.R;
    const int line = (int)(local % L), c16 = (int)(local / L);
    const bool live = line < J.lines;
    const int ex = live ? scale_exponent(J.maxabs[line]) : 0;
    if (J.exp_out && c16 == 0 && live) J.exp_out[line] = ex;
    int8_t out[kOzSlices][16];
#pragma unroll
    for (int x = 0; x < 16; ++x) {
      const int k = c16 * 16 + x;
      double y = (live && k < J.K) ? src[(long long)line * J.s_line + (long long)k * J.s_k] : 0.0;
      y = ldexp(y, -ex);
#pragma unroll
      for (int p = 0; p < kOzSlices; ++p) {
        y *= 128.0;
        const double a = rint(y);
        out[p][x] = (int8_t)a;
        y -= a;
      }
    }
    const int t = line / J.R, lr = line % J.R;
    uint8_t *base = J.dst + (long long)t * J.tile_stride +
                    oz_offset(J.R, 0, lr, (J.kb0 * kOzKBlock) + c16 * 16);
#pragma unroll
    for (int p = 0; p < kOzSlices; ++p) {
      int4 w;
      memcpy(&w, out[p], 16);
      *reinterpret_cast<int4 *>(base + (long long)p * J.R * kOzKBlock) = w;
    }
  }
}

int grid_for(long long threads) {
  const long long cap = (long long)num_sms() * 8;
  return (int)std::max(1LL, std::min(cap, (threads + 255) / 256));
}

}  // namespace

void ozaki_gemm(const OzSeg *d_segs, const OzTile *d_tiles, int ntiles, double *cbase,
                int *d_status, cudaStream_t stream) {
  if (ntiles <= 0) return;
  static bool configured = false;
  if (!configured) {
    HB_CUDA(cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmem));
    configured = true;
  }
  const int grid = std::min(ntiles, num_sms());
  ozaki_gemm_kernel<<<grid, kThreads, kSmem, stream>>>(d_segs, d_tiles, ntiles, cbase, d_status);
  HB_LAUNCHED();
}

long long ozaki_prepare_max(std::vector<MaxJob> &jobs) {
  long long items = 0;
  for (auto &j : jobs) {
    j.item0 = items;
    items += (j.s_k == 1) ? j.lines : (j.lines + 31) / 32;
  }
  return items;
}

long long ozaki_prepare_slice(std::vector<SliceJob> &jobs) {
  long long items = 0;
  for (auto &j : jobs) {
    HB_REQUIRE(j.R % 8 == 0 && j.R >= 8, INPUT_ERROR, "slice tile lines");
    j.item0 = items;
    items += (long long)j.ntiles * j.R * j.nkb * 2;
  }
  return items;
}

void ozaki_max(const MaxJob *d_jobs, int njobs, long long items, const double *xbase,
               cudaStream_t stream) {
  if (njobs <= 0 || items <= 0) return;
  max_kernel<<<grid_for(items * 32), 256, 0, stream>>>(d_jobs, njobs, items, xbase);
  HB_LAUNCHED();
}

void ozaki_slice(const SliceJob *d_jobs, int njobs, long long items, const double *xbase,
                 cudaStream_t stream) {
  if (njobs <= 0 || items <= 0) return;
  slice_kernel<<<grid_for(items), 256, 0, stream>>>(d_jobs, njobs, items, xbase);
  HB_LAUNCHED();
}

}  // namespace hb
