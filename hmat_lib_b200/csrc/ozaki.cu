// int8-sliced FP64 products on tcgen05 (see ozaki.h for the scheme and the
// blocked operand layout).
//
// Persistent kernel, one CTA of ten warps per SM, each taking the run of
// tiles the host schedule gave it (ozaki_schedule):
//   warp 0               producer: per K-block the A block (all S slices of
//                        128 lines) and the B block, each as 1-8 bulk copies
//                        issued by as many lanes, into a six-stage ring,
//                        completion on full[stage]; the next tile's
//                        descriptors are fetched while a tile streams;
//   warp 1 (one thread)  MMA issuer: per K-block the S(S+1)/2 slice products
//                        as 8 MMAs (slice p of A against slices q = 1 .. S+1-p
//                        of B, which sit next to each other in shared memory,
//                        so one MMA of N = (S+1-p) nw covers accumulator groups
//                        t = p + q - 2 stored side by side in TMEM), commit to
//                        empty[stage]; after the tile's last K-block a commit
//                        to tmem_full;
//   warps 2-9            epilogue (two warps per quarter of the TMEM lanes,
//                        alternate 16-column chunks): wait tmem_full, read the
//                        S int32 groups of their 32 lanes, combine them (each
//                        triple exactly in 64-bit integers, the two triples
//                        in FP64), release the accumulators (tmem_empty),
//                        then scale by
//                        2^(e_r + f_j) and store or atomically add the tile
//                        while the next tile's MMAs run.
// Warp 1 also owns the TMEM allocation (512 columns: S groups of <= 64).
// Every barrier wait is bounded; a wait that runs out sets the CTA's abort
// flag, every role leaves its loop, the producer waits (bounded) for its
// copies in flight, the MMA thread for its MMAs, and the kernel reports
// status 1 and returns.
#include <algorithm>
#include <cmath>
#include <queue>
#include <utility>
#include <vector>

#include "ozaki.h"
#include "umma.cuh"

namespace hb {

namespace {

constexpr int kEpiWarps = 8;                          // two per TMEM lane quarter
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr int kStages = 6;
constexpr int kStageBytes = kOzABlock + oz_bblock(kOzMaxNw);   // 36864
constexpr size_t kSmem = (size_t)kStages * kStageBytes;        // 221184
constexpr long long kWaitTries = 1LL << 26;
constexpr int kSliceBytesA = kOzRowsA * kOzKBlock;              // 4096: one slice of an A block

// 64-bit integer of magnitude below 2^51 -> double, exactly: adding it to
// the bit pattern of 1.5 2^52 gives the double 1.5 2^52 + x, so one integer
// addition and one subtraction replace the 64-bit conversion instruction.
__device__ __forceinline__ double exact_double46(long long x) {
  return __longlong_as_double(x + 0x4338000000000000LL) - 0x1.8p52;
}

// Bounded wait that also gives up when another role has aborted.
__device__ __forceinline__ bool wait_or_abort(uint64_t *bar, uint32_t parity, volatile int *bad) {
  for (long long i = 0; i < kWaitTries; ++i) {
    if (umma::mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && *bad) return false;
  }
  return false;
}

__global__ void __launch_bounds__(kThreads, 1)
ozaki_gemm_kernel(const OzSeg *__restrict__ segs, const OzTile *__restrict__ tiles,
                  const int *__restrict__ starts, double *cbase, int *status, int split) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(8) uint64_t empty[kStages];
  __shared__ __align__(8) uint64_t tmem_full, tmem_empty, mma_done;
  __shared__ uint32_t taddr_s;
  __shared__ volatile int bad;
  __shared__ int cexp_s[kEpiWarps][kOzMaxNw];   // per epilogue warp: column exponents of its tile
  static_assert(kOzSlices == 6, "the epilogue reads the groups in two passes of three");

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
    umma::mbar_init(&tmem_empty, kEpiWarps);
    umma::mbar_init(&mma_done, 1);
    umma::fence_mbar_init();
    bad = 0;
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = taddr_s;
  const int tile_first = starts[blockIdx.x], tile_end = starts[blockIdx.x + 1];

  if (warp == 0) {
    // ---------------- producer ----------------
    // lane 0 waits for a free stage and announces its bytes; lanes 0 .. split-1
    // then each copy 1/split of the A block and of the B block
    long long g = 0;   // K-blocks issued by this CTA
    bool stop = false;
    // descriptors run one tile ahead: the next tile's OzTile is loaded when a
    // tile starts and its segment descriptors (one per lane, nseg <= 32) after
    // the tile's first K-block is issued, so no descriptor load stalls the
    // ring at a tile or segment boundary
    OzTile T{};
    OzSeg Gl{};
    if (tile_first < tile_end) {
      T = tiles[tile_first];
      if (lane < T.nseg) Gl = segs[T.seg0 + lane];
    }
    for (int tile = tile_first; tile < tile_end && !stop; ++tile) {
      stop = __shfl_sync(0xffffffffu, (int)bad, 0) != 0;
      if (stop) break;
      const bool more = tile + 1 < tile_end;
      OzTile Tn{};
      if (more) Tn = tiles[tile + 1];
      OzSeg Gn{};
      bool next_segs = !more;
      const uint32_t bbytes = (uint32_t)oz_bblock(T.nw);
      const uint32_t ca = (uint32_t)kOzABlock / split, cb = bbytes / split;
      for (int q = 0; q < T.nseg && !stop; ++q) {
        const uint8_t *ga = (const uint8_t *)__shfl_sync(0xffffffffu, (unsigned long long)Gl.a, q);
        const uint8_t *gb = (const uint8_t *)__shfl_sync(0xffffffffu, (unsigned long long)Gl.b, q);
        const int nkb = __shfl_sync(0xffffffffu, Gl.nkb, q);
        for (int kb = 0; kb < nkb; ++kb) {
          const int st = (int)(g % kStages);
          const long long use = g / kStages;
          int ok = 1;
          if (lane == 0 && use > 0)
            ok = wait_or_abort(&empty[st], (uint32_t)((use - 1) & 1), &bad) ? 1 : 0;
          ok = __shfl_sync(0xffffffffu, ok, 0);
          if (!ok) {
            if (lane == 0) bad = 1;
            stop = true;
            break;
          }
          uint8_t *dst = sm + st * kStageBytes;
          if (lane == 0) umma::mbar_expect_tx(&full[st], (uint32_t)kOzABlock + bbytes);
          __syncwarp();
          if (lane < split) {
            umma::bulk_g2s(dst + lane * ca, ga + (long long)kb * kOzABlock + lane * ca, ca,
                           &full[st]);
            umma::bulk_g2s(dst + kOzABlock + lane * cb, gb + (long long)kb * bbytes + lane * cb,
                           cb, &full[st]);
          }
          ++g;
          if (!next_segs) {
            if (lane < Tn.nseg) Gn = segs[Tn.seg0 + lane];
            next_segs = true;
          }
        }
      }
      if (!next_segs && lane < Tn.nseg) Gn = segs[Tn.seg0 + lane];
      T = Tn;
      Gl = Gn;
    }
    // copies still in flight land before the CTA may exit
    if (lane == 0)
      for (long long q = std::max(0LL, g - kStages); q < g; ++q)
        umma::mbar_wait_bounded(&full[q % kStages], (uint32_t)((q / kStages) & 1), kWaitTries);
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      long long g = 0;
      int lt = 0;
      bool ok = true;
      OzTile Tn{};
      if (tile_first < tile_end) Tn = tiles[tile_first];
      for (int tile = tile_first; tile < tile_end && ok && !bad; ++tile, ++lt) {
        const OzTile T = Tn;
        if (tile + 1 < tile_end) Tn = tiles[tile + 1];   // lands while this tile runs
        if (lt > 0 && !wait_or_abort(&tmem_empty, (uint32_t)((lt - 1) & 1), &bad)) {
          ok = false;
          break;
        }
        umma::fence_after_sync();
        const int nw = T.nw;
        const int maxcnt = min(kOzSlices, 256 / nw);
        const uint32_t bslice = (uint32_t)nw * kOzKBlock;
        bool first = true;
        {
          for (int kb = 0; kb < T.nkb; ++kb, ++g) {
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
    const int ew = warp - 2;        // epilogue warp 0 .. kEpiWarps - 1
    const int half = ew >> 2;       // the two warps of a quarter take alternate 16-column chunks
    const uint32_t lane_addr = tbase + ((uint32_t)(32 * quarter) << 16);
    const int r = 32 * quarter + lane;
    int lt = 0;
    for (int tile = tile_first; tile < tile_end; ++tile, ++lt) {
      if (__any_sync(0xffffffffu, bad)) break;
      const OzTile T = tiles[tile];
      // column exponents of this tile, staged while its MMAs run
      __syncwarp();
      for (int j = lane; j < kOzMaxNw; j += 32) cexp_s[ew][j] = j < T.cols ? T.cexp[j] : 0;
      __syncwarp();
      const bool ready = wait_or_abort(&tmem_full, (uint32_t)(lt & 1), &bad);
      if (!__all_sync(0xffffffffu, ready)) {
        bad = 1;
        break;
      }
      umma::fence_after_sync();
      const int nw = T.nw;
      const bool row_ok = r < T.rows;
      // 2^14 sum_t v_t 2^(-7 t) of the (at most two) 16-column chunks of
      // this warp, held in registers so that the accumulators go back to the
      // MMA thread before the tile is scaled and stored.  Each triple of
      // groups is combined exactly in 64-bit integers (|.| < 2^46), converted
      // exactly, and the two triples are added with one rounding.
      double acc[2][16];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int c0 = 16 * half + 32 * c;
        if (c0 < nw) {
          // two passes of three groups (lowest first) keep 48 int registers
          // live beside the 32 accumulating doubles
#pragma unroll
          for (int pass = 0; pass < 2; ++pass) {
            int32_t v[3][16];
#pragma unroll
            for (int u = 0; u < 3; ++u)
              umma::tmem_ld16(lane_addr + (3 * (1 - pass) + u) * nw + c0, v[u]);
            umma::tmem_ld_wait();
#pragma unroll
            for (int x = 0; x < 16; ++x) {
              const long long tri =
                  (long long)v[0][x] * 16384 + (long long)v[1][x] * 128 + (long long)v[2][x];
              const double d = exact_double46(tri);
              acc[c][x] = pass == 0 ? d : fma(acc[c][x], 0x1p-21, d);
            }
          }
        }
      }
      umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) umma::mbar_arrive(&tmem_empty);
      // the common factor 2^(e_r + f_j - 28), then store or add
      if (row_ok) {
        const int er = T.rexp[r] - 28;
        double *crow = cbase + T.c_off + r;
        double rowmax = 0.0;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int c0 = 16 * half + 32 * c;
#pragma unroll
          for (int x = 0; x < 16; ++x) {
            const int j = c0 + x;
            if (c0 < nw && j < T.cols) {
              const int e = er + cexp_s[ew][j];
              const double val = (e >= -1022 && e <= 1023)
                                     ? acc[c][x] * __longlong_as_double((long long)(e + 1023) << 52)
                                     : ldexp(acc[c][x], e);
              rowmax = fmax(rowmax, fabs(val));
              double *cp = crow + (long long)j * T.ldc;
              if (T.atomic)
                atomicAdd(cp, val);
              else
                *cp = val;
            }
          }
        }
        if (T.rmax && rowmax > 0.0)
          atomicMax(T.rmax + r, (unsigned long long)__double_as_longlong(rowmax));
      }
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

constexpr int kMaxChunkK = 1024;   // K values per warp item, K-contiguous lines
constexpr int kMaxChunkL = 16;     // K values per warp item, line-contiguous (32 lines)
constexpr int kTileLines = 32;     // shared-memory transpose tile: lines x K values
constexpr int kTileK = 64;
constexpr int kSliceThreads = kTileLines * (kTileK / 16);   // one (line, 16-value chunk) each

__device__ __forceinline__ void max_into(unsigned long long *out, double mx) {
  if (mx > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(mx));
}

// Work items are warps: one line and kMaxChunkK of its K values (K
// contiguous: lanes split K), or 32 lines (one per lane) and kMaxChunkL K
// values.
__global__ void max_kernel(const MaxJob *__restrict__ jobs, int njobs, long long items,
                           const double *xbase) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long it = w0; it < items; it += nwarps) {
    const MaxJob &J = jobs[find_job(jobs, njobs, it)];
    const double *src = J.src ? J.src : xbase;
    const long long local = it - J.item0;
    double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
    if (J.s_k == 1) {
      const int nch = (J.K + kMaxChunkK - 1) / kMaxChunkK;
      const long long line = local / nch;
      const int k0 = (int)(local % nch) * kMaxChunkK, k1 = min(J.K, k0 + kMaxChunkK);
      const double *row = src + line * J.s_line;
      int k = k0 + lane;
      for (; k + 224 < k1; k += 256) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = row[k + 32 * u];
        m0 = fmax(m0, fmax(fabs(v[0]), fabs(v[1])));
        m1 = fmax(m1, fmax(fabs(v[2]), fabs(v[3])));
        m2 = fmax(m2, fmax(fabs(v[4]), fabs(v[5])));
        m3 = fmax(m3, fmax(fabs(v[6]), fabs(v[7])));
      }
      for (; k < k1; k += 32) m0 = fmax(m0, fabs(row[k]));
      double mx = fmax(fmax(m0, m1), fmax(m2, m3));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) max_into(J.out + line, mx);
    } else {
      const int nch = (J.K + kMaxChunkL - 1) / kMaxChunkL;
      const long long line = (local / nch) * 32 + lane;
      const int k0 = (int)(local % nch) * kMaxChunkL, k1 = min(J.K, k0 + kMaxChunkL);
      if (line < J.lines) {
        const double *p = src + line * J.s_line;
        int k = k0;
        for (; k + 3 < k1; k += 4) {
          m0 = fmax(m0, fabs(p[(long long)k * J.s_k]));
          m1 = fmax(m1, fabs(p[(long long)(k + 1) * J.s_k]));
          m2 = fmax(m2, fabs(p[(long long)(k + 2) * J.s_k]));
          m3 = fmax(m3, fabs(p[(long long)(k + 3) * J.s_k]));
        }
        for (; k < k1; ++k) m0 = fmax(m0, fabs(p[(long long)k * J.s_k]));
        max_into(J.out + line, fmax(fmax(m0, m1), fmax(m2, m3)));
      }
    }
  }
}

// Six slices of 16 consecutive K values of one line, stored as six aligned
// 16-byte words at `base` + p R 32.  Each value is rounded once to the
// integer N = x 2^(42 - ex) (|N| <= 127 2^35 because |x| 2^-ex <= 127/128)
// and written in balanced base 128, N = sum_p d_p 128^(6-p): with
// M = N + 2^42 + 64 (128^4 + ... + 1) >= 0, d_p = digit_p(M) - 64 for p > 1
// (in [-64, 63]) and d_1 = (M >> 35) - 128 (in [-127, 127]).
__device__ __forceinline__ void slice16(const double (&y0)[16], int ex, uint8_t *base, int R) {
  constexpr long long kBias = (1LL << 42) + 64LL * ((1LL << 28) + (1LL << 21) + (1LL << 14) +
                                                    (1LL << 7) + 1LL);
  const int sh = 42 - ex;
  const bool fast = sh >= -1022 && sh <= 1023;
  const double scale = fast ? __longlong_as_double((long long)(sh + 1023) << 52) : 0.0;
  uint32_t w[kOzSlices][4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t b[kOzSlices] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      const double v = y0[4 * q + x];
      const long long N = __double2ll_rn(fast ? v * scale : ldexp(v, sh));
      const unsigned long long M = (unsigned long long)(N + kBias);
      const uint32_t lo = (uint32_t)M;                  // digits 4..6 (bits 0..20) and part of 3
      const uint32_t hi = (uint32_t)(M >> 21);          // digits 1..3
      const uint32_t d[kOzSlices] = {((hi >> 14) - 128u) & 0xFFu, (((hi >> 7) & 127u) - 64u) & 0xFFu,
                                     ((hi & 127u) - 64u) & 0xFFu, (((lo >> 14) & 127u) - 64u) & 0xFFu,
                                     (((lo >> 7) & 127u) - 64u) & 0xFFu, ((lo & 127u) - 64u) & 0xFFu};
#pragma unroll
      for (int p = 0; p < kOzSlices; ++p) b[p] |= d[p] << (8 * x);
    }
#pragma unroll
    for (int p = 0; p < kOzSlices; ++p) w[p][q] = b[p];
  }
#pragma unroll
  for (int p = 0; p < kOzSlices; ++p)
    *reinterpret_cast<uint4 *>(base + (long long)p * R * kOzKBlock) =
        make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
}

// Line-contiguous sources: one item = 16 consecutive K positions of one
// line; lines vary fastest, so loads are coalesced and eight neighbouring
// items fill one 128-byte core matrix.
__global__ void slice_lines_kernel(const SliceJob *__restrict__ jobs, int njobs, long long items,
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
    double y[16];
#pragma unroll
    for (int x = 0; x < 16; ++x) {
      const int k = c16 * 16 + x;
      y[x] = (live && k < J.K) ? src[(long long)line * J.s_line + (long long)k * J.s_k] : 0.0;
    }
    const int t = line / J.R, lr = line % J.R;
    slice16(y, ex, J.dst + (long long)t * J.tile_stride +
                       oz_offset(J.R, 0, lr, J.kb0 * kOzKBlock + c16 * 16), J.R);
  }
}

// 8-byte asynchronous copy into shared memory; bytes = 0 writes zeros (the
// source address is then not read).
__device__ __forceinline__ void cp_async8z(void *smem, const void *gmem, bool pred) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem),
               "r"(pred ? 8 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_prev() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// Stages block item `it` (32 lines x 64 K values) of a K-contiguous slice
// batch into `buf` with asynchronous copies (zeros outside the source).
__device__ __forceinline__ void stage_kcontig(const SliceJob *__restrict__ jobs, int njobs,
                                              long long it, const double *xbase,
                                              double (*buf)[kTileK + 1]) {
  const SliceJob &J = jobs[find_job(jobs, njobs, it)];
  const double *src = J.src ? J.src : xbase;
  const long long local = it - J.item0;
  const int Kw = J.nkb * kOzKBlock;
  const int nkt = (Kw + kTileK - 1) / kTileK;
  const int line0 = (int)(local / nkt) * kTileLines, k0 = (int)(local % nkt) * kTileK;
  for (int idx = threadIdx.x; idx < kTileLines * kTileK; idx += blockDim.x) {
    const int l = idx / kTileK, kk = idx % kTileK;
    const int line = line0 + l, k = k0 + kk;
    const bool in = line < J.lines && k < J.K;
    cp_async8z(&buf[l][kk], in ? src + (long long)line * J.s_line + k : src, in);
  }
}

// K-contiguous sources (s_k = 1): one block item = 32 lines x 64 K values,
// brought into shared memory with coalesced asynchronous row copies (the next
// item's copies in flight while the current one is sliced, two buffers),
// then sliced 16 K values per thread.
__global__ void __launch_bounds__(kSliceThreads) slice_kcontig_kernel(const SliceJob *__restrict__ jobs,
                                                            int njobs, long long items,
                                                            const double *xbase) {
  __shared__ double buf[2][kTileLines][kTileK + 1];
  const int tid = threadIdx.x;
  long long it = blockIdx.x;
  if (it < items) stage_kcontig(jobs, njobs, it, xbase, buf[0]);
  cp_async_commit_group();
  for (int b = 0; it < items; it += gridDim.x, b ^= 1) {
    if (it + gridDim.x < items) stage_kcontig(jobs, njobs, it + gridDim.x, xbase, buf[b ^ 1]);
    cp_async_commit_group();
    cp_async_wait_prev();            // this item's group has landed
    __syncthreads();
    const SliceJob &J = jobs[find_job(jobs, njobs, it)];
    const long long local = it - J.item0;
    const int Kw = J.nkb * kOzKBlock;                   // K positions written
    const int nkt = (Kw + kTileK - 1) / kTileK;
    const int line0 = (int)(local / nkt) * kTileLines, k0 = (int)(local % nkt) * kTileK;
    const int l = tid % kTileLines, c = tid / kTileLines;   // kTileK / 16 chunks
    const int line = line0 + l, k = k0 + c * 16;
    if (line < J.ntiles * J.R && k < Kw) {
      const bool live = line < J.lines;
      const int ex = live ? scale_exponent(J.maxabs[line]) : 0;
      if (J.exp_out && k == 0 && live) J.exp_out[line] = ex;
      double y[16];
#pragma unroll
      for (int x = 0; x < 16; ++x) y[x] = buf[b][l][c * 16 + x];
      const int t = line / J.R, lr = line % J.R;
      slice16(y, ex, J.dst + (long long)t * J.tile_stride +
                         oz_offset(J.R, 0, lr, J.kb0 * kOzKBlock + k), J.R);
    }
    __syncthreads();                 // buf[b] is refilled two items later
  }
}

__global__ void ranges_kernel(const CopyRange *__restrict__ ranges) {
  const CopyRange R = ranges[blockIdx.y];
  auto *d = (unsigned long long *)R.dst;
  auto *src = (const unsigned long long *)R.src;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < R.words;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = src ? src[i] : 0ULL;
}

int grid_for(long long threads) {
  const long long cap = (long long)num_sms() * 8;
  return (int)std::max(1LL, std::min(cap, (threads + 255) / 256));
}

}  // namespace

int ozaki_grid(int ntiles) { return std::max(0, std::min(ntiles, num_sms())); }

std::vector<int> ozaki_schedule(std::vector<OzTile> &tiles, const std::vector<OzSeg> &segs,
                                int grid) {
  std::vector<int> start(grid + 1, 0);
  if (grid <= 0 || tiles.empty()) {
    std::fill(start.begin(), start.end(), (int)tiles.size());
    if (!start.empty()) start[0] = 0;
    return start;
  }
  // cost in K-block x column units; the fixed part is about two K-blocks of
  // a 64-wide tile (the wait for the accumulators between tiles)
  constexpr long long kTileCost = 160;
  std::vector<long long> cost(tiles.size());
  for (size_t i = 0; i < tiles.size(); ++i) {
    HB_REQUIRE(tiles[i].nseg >= 0 && tiles[i].nseg <= 32, INPUT_ERROR,
               "int8 product: more than 32 segments in a tile");
    long long kb = 0;
    for (int q = tiles[i].seg0; q < tiles[i].seg0 + tiles[i].nseg; ++q) kb += segs[q].nkb;
    HB_REQUIRE(kb < (1LL << 31), INPUT_ERROR, "int8 product: K range too long");
    tiles[i].nkb = (int)kb;
    cost[i] = kb * tiles[i].nw + kTileCost;
  }
  std::vector<int> order(tiles.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  if (option("ozaki_schedule", 1.0) == 0.0) {
    // option ozaki_schedule = 0: tile i on CTA i mod grid, in list order
    std::vector<OzTile> out;
    out.reserve(tiles.size());
    for (int b = 0; b < grid; ++b) {
      start[b] = (int)out.size();
      for (size_t i = b; i < tiles.size(); i += grid) out.push_back(tiles[i]);
    }
    start[grid] = (int)out.size();
    tiles.swap(out);
    return start;
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  // least-loaded CTA first (ties: lower index)
  using Slot = std::pair<long long, int>;
  std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
  for (int b = 0; b < grid; ++b) heap.push({0, b});
  std::vector<std::vector<int>> owned(grid);
  for (int i : order) {
    Slot sl = heap.top();
    heap.pop();
    owned[sl.second].push_back(i);
    heap.push({sl.first + cost[i], sl.second});
  }
  std::vector<OzTile> out;
  out.reserve(tiles.size());
  for (int b = 0; b < grid; ++b) {
    start[b] = (int)out.size();
    for (int i : owned[b]) out.push_back(tiles[i]);
  }
  start[grid] = (int)out.size();
  tiles.swap(out);
  return start;
}

void ozaki_gemm(const OzSeg *d_segs, const OzTile *d_tiles, const int *d_starts, int grid,
                double *cbase, int *d_status, cudaStream_t stream) {
  if (grid <= 0) return;
  static bool configured = false;
  if (!configured) {
    HB_CUDA(cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSmem));
    configured = true;
  }
  // bulk copies per operand block (1, 2, 4 or 8 lanes; every chunk stays a
  // multiple of 16 bytes since B blocks are multiples of 384 bytes)
  int split = (int)option("ozaki_copy_split", 1.0);
  split = split >= 8 ? 8 : split >= 4 ? 4 : split >= 2 ? 2 : 1;
  ozaki_gemm_kernel<<<grid, kThreads, kSmem, stream>>>(d_segs, d_tiles, d_starts, cbase, d_status,
                                                       split);
  HB_LAUNCHED();
}

void ozaki_ranges(const CopyRange *d_ranges, int n, cudaStream_t stream) {
  for (int off = 0; off < n; off += 65535) {
    ranges_kernel<<<dim3(16, std::min(65535, n - off)), 256, 0, stream>>>(d_ranges + off);
    HB_LAUNCHED();
  }
}

MaxBatch ozaki_max_batch(std::vector<MaxJob> jobs, cudaStream_t stream) {
  MaxBatch b;
  for (auto &j : jobs) {
    j.item0 = b.items;
    b.items += (j.s_k == 1) ? (long long)j.lines * ((j.K + kMaxChunkK - 1) / kMaxChunkK)
                            : (long long)((j.lines + 31) / 32) * ((j.K + kMaxChunkL - 1) / kMaxChunkL);
  }
  b.n = (int)jobs.size();
  if (b.n) {
    HB_CUDA(cudaMalloc((void **)&b.d, sizeof(MaxJob) * jobs.size()));
    HB_CUDA(cudaMemcpyAsync(b.d, jobs.data(), sizeof(MaxJob) * jobs.size(), cudaMemcpyHostToDevice,
                            stream));
  }
  return b;
}

SliceBatch ozaki_slice_batch(std::vector<SliceJob> jobs, cudaStream_t stream) {
  SliceBatch b;
  b.kcontig = !jobs.empty() && jobs[0].s_k == 1;
  for (auto &j : jobs) {
    HB_REQUIRE(j.R % 8 == 0 && j.R >= 8, INPUT_ERROR, "slice tile lines");
    HB_REQUIRE((j.s_k == 1) == b.kcontig, INPUT_ERROR, "mixed slice job kinds in one batch");
    j.item0 = b.items;
    const long long L = (long long)j.ntiles * j.R;
    b.items += b.kcontig ? ((L + kTileLines - 1) / kTileLines) *
                               ((j.nkb * kOzKBlock + kTileK - 1) / kTileK)
                         : L * j.nkb * 2;
  }
  b.n = (int)jobs.size();
  if (b.n) {
    HB_CUDA(cudaMalloc((void **)&b.d, sizeof(SliceJob) * jobs.size()));
    HB_CUDA(cudaMemcpyAsync(b.d, jobs.data(), sizeof(SliceJob) * jobs.size(),
                            cudaMemcpyHostToDevice, stream));
  }
  return b;
}

void ozaki_max(const MaxBatch &b, const double *xbase, cudaStream_t stream) {
  if (b.n <= 0 || b.items <= 0) return;
  max_kernel<<<grid_for(b.items * 32), 256, 0, stream>>>(b.d, b.n, b.items, xbase);
  HB_LAUNCHED();
}

void ozaki_slice(const SliceBatch &b, const double *xbase, cudaStream_t stream) {
  if (b.n <= 0 || b.items <= 0) return;
  if (b.kcontig) {
    // two 16.6 KB buffers per block: six resident blocks per SM
    const int grid = (int)std::min<long long>(b.items, (long long)num_sms() * 6);
    slice_kcontig_kernel<<<grid, kSliceThreads, 0, stream>>>(b.d, b.n, b.items, xbase);
  } else {
    slice_lines_kernel<<<grid_for(b.items), 256, 0, stream>>>(b.d, b.n, b.items, xbase);
  }
  HB_LAUNCHED();
}

}  // namespace hb
