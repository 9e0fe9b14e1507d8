// FP64 variable-batched segmented GEMM for sm_100a.
//
// Two kernels (option gemm_f64_engine): the FP64 tensor-core (DMMA) kernel
// (default, below), and a CUDA-core DFMA kernel: 256 threads, a BM x BN output tile per CTA
// (128 x 64, 64 x 128, 32 x 128 or 32 x 256), K advanced 16 at a time through a two-stage
// cp.async pipeline (8-byte copies with zero fill, so any leading dimension
// and any offset work), 32 accumulators per thread, operands read from shared
// memory as double2.  FP64 has no tcgen05 path; this is the FP64 roofline
// kernel (B200: 64 DFMA / clock / SM).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>

#include "gemm_f64.h"

namespace hb {

int gemm_f64_engine() { return (int)option("gemm_f64_engine", 2); }

double &gemm_flops_counter() {
  static thread_local double flops = 0.0;
  return flops;
}

double &plan_host_ms() {
  static thread_local double ms = 0.0;
  return ms;
}

namespace {

constexpr int kBK = 16;
constexpr int kThreads = 256;

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// bases.p[i] for a runtime i without copying the launch argument array to
// local memory (a chain of selects on the constant-bank values)
__device__ __forceinline__ double *base_ptr(const GemmBases &b, int i) {
  static_assert(kGemmBases == 6, "base_ptr selects among six slots");
  double *p = b.p[0];
  p = i == 1 ? b.p[1] : p;
  p = i == 2 ? b.p[2] : p;
  p = i == 3 ? b.p[3] : p;
  p = i == 4 ? b.p[4] : p;
  p = i == 5 ? b.p[5] : p;
  return p;
}

struct KIter {
  int si;      // segment index (absolute)
  int kk;      // position inside the segment
  int le;      // end of the valid range inside the segment
  int kbase;   // concatenated-K position of the segment start
};

template <int BM, int BN>
struct Smem {
  static constexpr int LDA = BM + 2;
  static constexpr int LDB = BN + 2;
  static constexpr size_t bytes = sizeof(double) * 2 * kBK * (LDA + LDB);
};

template <int BM, int BN>
__global__ void __launch_bounds__(kThreads, 2)
gemm_f64_kernel(const GemmSeg *__restrict__ segs, const GemmProb *__restrict__ probs,
                const GemmTile *__restrict__ tiles, GemmBases bases) {
  constexpr int TM = BM / 16, TN = BN / 16;
  constexpr int LDA = Smem<BM, BN>::LDA, LDB = Smem<BM, BN>::LDB;
  extern __shared__ __align__(16) double smem[];
  double *As = smem;                        // [2][kBK][LDA]
  double *Bs = smem + 2 * kBK * LDA;        // [2][kBK][LDB]

  const GemmTile tile = tiles[blockIdx.x];
  const GemmProb P = probs[tile.prob];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int seg_end = P.seg0 + P.nseg;

  double acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;

  auto settle = [&](KIter &it) {
    while (it.si < seg_end) {
      const int K = segs[it.si].K;
      const int ls = max(tile.k0 - it.kbase, 0);
      const int le = min(tile.k1 - it.kbase, K);
      if (ls < le) {
        it.kk = ls;
        it.le = le;
        return;
      }
      it.kbase += K;
      ++it.si;
    }
  };
  auto advance = [&](KIter &it) {
    it.kk += kBK;
    if (it.kk >= it.le) {
      it.kbase += segs[it.si].K;
      ++it.si;
      settle(it);
    }
  };

  // One operand element into shared memory: copied from global memory, or
  // computed when the segment's operand is a generated kernel matrix (stored
  // element (row, col) of the block at gen_offset(row0, col0)).
  auto stage = [&](double *dst, bool gen, const double *base, long long off, long long row,
                   long long col, long long ld, bool p) {
    if (gen) {
      *dst = p ? kernel_entry(bases.gen, (int)(off >> 32) + (int)row,
                              (int)(off & 0xffffffffLL) + (int)col)
               : 0.0;
    } else {
      cp_async8(dst, p ? base + off + row + col * ld : base, p);
    }
  };

  auto load = [&](int buf, const KIter &it) {
    const GemmSeg S = segs[it.si];
    const bool ga = S.abase == kGenSlot, gb = S.bbase == kGenSlot;
    const double *A = ga ? nullptr : base_ptr(bases, S.abase);
    const double *B = gb ? nullptr : base_ptr(bases, S.bbase);
    double *as = As + buf * kBK * LDA;
    double *bs = Bs + buf * kBK * LDB;
    const int kk = it.kk, kend = it.le;
    if (S.ta == 0) {
      constexpr int KS = kThreads / BM;
      const int m = tid % BM;
      const bool mok = (tile.m0 + m) < P.M;
#pragma unroll
      for (int i = 0; i < BM * kBK / kThreads; ++i) {
        const int k = tid / BM + KS * i;
        const bool p = mok && (kk + k) < kend;
        stage(as + k * LDA + m, ga, A, S.a_off, tile.m0 + m, kk + k, S.lda, p);
      }
    } else {
      const int k = tid & 15;
      const bool kok = (kk + k) < kend;
#pragma unroll
      for (int i = 0; i < BM / 16; ++i) {
        const int m = (tid >> 4) + 16 * i;
        const bool p = kok && (tile.m0 + m) < P.M;
        stage(as + k * LDA + m, ga, A, S.a_off, kk + k, tile.m0 + m, S.lda, p);
      }
    }
    if (S.tb == 0) {
      const int k = tid & 15;
      const bool kok = (kk + k) < kend;
#pragma unroll
      for (int i = 0; i < BN / 16; ++i) {
        const int n = (tid >> 4) + 16 * i;
        const bool p = kok && (tile.n0 + n) < P.N;
        stage(bs + k * LDB + n, gb, B, S.b_off, kk + k, tile.n0 + n, S.ldb, p);
      }
    } else {
      constexpr int KS = kThreads / BN;
      const int n = tid % BN;
      const bool nok = (tile.n0 + n) < P.N;
#pragma unroll
      for (int i = 0; i < BN * kBK / kThreads; ++i) {
        const int k = tid / BN + KS * i;
        const bool p = nok && (kk + k) < kend;
        stage(bs + k * LDB + n, gb, B, S.b_off, tile.n0 + n, kk + k, S.ldb, p);
      }
    }
  };

  KIter it{P.seg0, 0, 0, 0};
  settle(it);
  int buf = 0;
  if (it.si < seg_end) load(0, it);
  cp_async_commit();
  while (it.si < seg_end) {
    KIter nx = it;
    advance(nx);
    if (nx.si < seg_end) load(buf ^ 1, nx);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const double *as = As + buf * kBK * LDA;
    const double *bs = Bs + buf * kBK * LDB;
#pragma unroll
    for (int k = 0; k < kBK; ++k) {
      double a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < TM / 2; ++i) {
        const double2 v = *reinterpret_cast<const double2 *>(as + k * LDA + 2 * ty + 32 * i);
        a[2 * i] = v.x;
        a[2 * i + 1] = v.y;
      }
#pragma unroll
      for (int j = 0; j < TN / 2; ++j) {
        const double2 v = *reinterpret_cast<const double2 *>(bs + k * LDB + 2 * tx + 32 * j);
        b[2 * j] = v.x;
        b[2 * j + 1] = v.y;
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
    buf ^= 1;
    it = nx;
  }
  cp_async_wait<0>();

  double *C = base_ptr(bases, P.cbase) + P.c_off;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int m = tile.m0 + 2 * ty + 32 * (i >> 1) + (i & 1);
    if (m >= P.M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int n = tile.n0 + 2 * tx + 32 * (j >> 1) + (j & 1);
      if (n >= P.N) continue;
      double *c = C + m + (long long)n * P.ldc;
      const double v = P.alpha * acc[i][j];
      if (P.split > 1)
        atomicAdd(c, v);
      else
        *c = (P.beta == 0.0) ? v : v + P.beta * (*c);
    }
  }
}

// ---- FP64 tensor-core (DMMA) variant ------------------------------------------------
// Same tiles, segments and K iteration as gemm_f64_kernel, with the multiply-adds
// on the FP64 tensor-core path (mma.sync m8n8k4 .f64: one warp instruction is an
// 8 x 8 x 4 product, 256 FMAs).  Eight warps per CTA, each owning a WM x WN
// sub-tile of the BM x BN output (WM/8 x WN/8 MMA tiles, two accumulators per
// lane each).  K advances BK (16 or 32: option gemm_f64_engine 1 / 2) at a time
// through a cp.async ring; 32-deep stages halve the per-stage work (copy set-up,
// barrier, segment bookkeeping) per MMA and were 10% faster on B200.  Each operand
// is staged in the layout that makes its global reads contiguous: an operand
// whose contiguous dimension is K is stored [row][k] (BK + 4 doubles per
// row), otherwise [k][row] (BM or BN + 4 per k); the pads make every fragment
// load of a half-warp hit 16 distinct 8-byte bank pairs.  Copies are 16 bytes
// when the operand's offset and leading dimension (and, for K-contiguous
// operands, the first K index) are even, else 8; elements past M, N or the K
// range are zero-filled.  The ring is as deep as two CTAs per SM allow (2 to
// 4 stages).
template <int BM, int BN, int BK>
struct MmaSmem {
  static constexpr int LDKM = BM + 4;      // [k][m] layout
  static constexpr int LDKN = BN + 4;      // [k][n] layout
  static constexpr int LDK = BK + 4;      // [m][k] / [n][k] layout
  static constexpr int A_ELEMS = (BK * LDKM > BM * LDK) ? BK * LDKM : BM * LDK;
  static constexpr int B_ELEMS = (BK * LDKN > BN * LDK) ? BK * LDKN : BN * LDK;
  static constexpr int STAGE = A_ELEMS + B_ELEMS;
  static constexpr int STAGES_FIT = (int)(112 * 1024 / (sizeof(double) * STAGE));
  static constexpr int STAGES = STAGES_FIT > 4 ? 4 : (STAGES_FIT < 2 ? 2 : STAGES_FIT);
  static constexpr size_t bytes = sizeof(double) * STAGES * STAGE;
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
               "r"(src_bytes));
}

__device__ __forceinline__ void dmma884(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

template <int BM, int BN, int WM, int WN, int BK>
__global__ void __launch_bounds__(kThreads, 2)
gemm_f64_mma_kernel(const GemmSeg *__restrict__ segs, const GemmProb *__restrict__ probs,
                    const GemmTile *__restrict__ tiles, GemmBases bases) {
  using SM = MmaSmem<BM, BN, BK>;
  constexpr int kMmaStages = SM::STAGES;
  constexpr int MT = WM / 8, NT = WN / 8;          // MMA tiles per warp
  constexpr int WARPS_N = BN / WN;
  static_assert((BM / WM) * (BN / WN) == kThreads / 32, "eight warps per CTA");
  extern __shared__ __align__(16) double smem[];

  const GemmTile tile = tiles[blockIdx.x];
  const GemmProb P = probs[tile.prob];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp / WARPS_N) * WM, wn0 = (warp % WARPS_N) * WN;
  const int seg_end = P.seg0 + P.nseg;

  double acc[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  auto settle = [&](KIter &it) {
    while (it.si < seg_end) {
      const int K = segs[it.si].K;
      const int ls = max(tile.k0 - it.kbase, 0);
      const int le = min(tile.k1 - it.kbase, K);
      if (ls < le) {
        it.kk = ls;
        it.le = le;
        return;
      }
      it.kbase += K;
      ++it.si;
    }
  };
  auto advance = [&](KIter &it) {
    it.kk += BK;
    if (it.kk >= it.le) {
      it.kbase += segs[it.si].K;
      ++it.si;
      settle(it);
    }
  };

  // One operand tile of `rows` lines (M or N side) x BK into stage memory.
  // `kcontig`: K is the contiguous dimension in global memory (stored
  // [line][k] in shared memory), otherwise lines are ([k][line]).  Element
  // (line, k) of the tile is global (row0 + line, kk + k) of the operand,
  // stored at base + off + r + c ld with (r, c) = (line, k), or (k, line) when
  // kcontig; lines >= nlines and k >= kend are zero.
  auto load_operand = [&](double *dst, bool gen, const double *base, long long off, long long ld,
                          bool kcontig, int rows, int row0, int nlines, int kk, int kend) {
    if (gen) {
      // generated kernel-matrix entries: (r, c) of the block at gen_offset(row0, col0)
      const int gr0 = (int)(off >> 32), gc0 = (int)(off & 0xffffffffLL);
      for (int e = tid; e < rows * BK; e += kThreads) {
        int line, k;
        if (kcontig) {
          line = e / BK;
          k = e % BK;
        } else {
          k = e / rows;
          line = e % rows;
        }
        const bool p = (row0 + line) < nlines && (kk + k) < kend;
        double v = 0.0;
        if (p) {
          const int r = kcontig ? kk + k : row0 + line;
          const int c = kcontig ? row0 + line : kk + k;
          v = kernel_entry(bases.gen, gr0 + r, gc0 + c);
        }
        if (kcontig)
          dst[line * SM::LDK + k] = v;
        else
          dst[k * (rows + 4) + line] = v;
      }
      return;
    }
    // 16-byte copies need even element offsets: the operand's offset and
    // leading dimension, and for K-contiguous operands the first K index
    const bool vec = ((off | ld | (kcontig ? kk : 0)) & 1) == 0 &&
                     (((unsigned long long)base) & 15) == 0;
    if (kcontig) {
      // per line BK contiguous K values: BK / 2 chunks of 16 bytes
      constexpr int CH = BK / 2;
      for (int e = tid; e < rows * CH; e += kThreads) {
        const int line = e / CH, k = 2 * (e % CH);
        const bool lok = (row0 + line) < nlines;
        const int nk = lok ? min(2, max(0, kend - (kk + k))) : 0;
        double *d = dst + line * SM::LDK + k;
        const double *src = base + off + (long long)(row0 + line) * ld + (kk + k);
        if (vec) {
          cp_async16(d, nk > 0 ? src : base, 8 * nk);
        } else {
          cp_async8(d, nk > 0 ? src : base, nk > 0);
          cp_async8(d + 1, nk > 1 ? src + 1 : base, nk > 1);
        }
      }
    } else {
      // per k, `rows` contiguous lines: rows / 2 chunks of 16 bytes
      const int CH = rows / 2;
      for (int e = tid; e < BK * CH; e += kThreads) {
        const int k = e / CH, line = 2 * (e % CH);
        const bool kok = (kk + k) < kend;
        const int nl = kok ? min(2, max(0, nlines - (row0 + line))) : 0;
        double *d = dst + k * (rows + 4) + line;
        const double *src = base + off + (row0 + line) + (long long)(kk + k) * ld;
        if (vec) {
          cp_async16(d, nl > 0 ? src : base, 8 * nl);
        } else {
          cp_async8(d, nl > 0 ? src : base, nl > 0);
          cp_async8(d + 1, nl > 1 ? src + 1 : base, nl > 1);
        }
      }
    }
  };

  // Stage `buf` <- K-block `it`; returns its layout bits (1: A stored [m][k],
  // 2: B stored [n][k]).
  auto load = [&](int buf, const KIter &it) -> int {
    const GemmSeg S = segs[it.si];
    const bool ga = S.abase == kGenSlot, gb = S.bbase == kGenSlot;
    double *as = smem + buf * SM::STAGE;
    double *bs = as + SM::A_ELEMS;
    // op(A) is M x K: ta = 0 stores (m, k) at m + k lda (lines contiguous),
    // ta = 1 stores it at k + m lda (K contiguous)
    load_operand(as, ga, ga ? nullptr : base_ptr(bases, S.abase), S.a_off, S.lda, S.ta == 1, BM,
                 tile.m0, P.M, it.kk, it.le);
    // op(B) is K x N: tb = 0 stores (k, n) at k + n ldb (K contiguous),
    // tb = 1 at n + k ldb (lines contiguous)
    load_operand(bs, gb, gb ? nullptr : base_ptr(bases, S.bbase), S.b_off, S.ldb, S.tb == 0, BN,
                 tile.n0, P.N, it.kk, it.le);
    return (S.ta == 1 ? 1 : 0) | (S.tb == 0 ? 2 : 0);
  };

  // ring of kMmaStages buffers; `lay` keeps 2 layout bits per buffer
  KIter it{P.seg0, 0, 0, 0};
  settle(it);
  unsigned lay = 0;
#pragma unroll
  for (int st = 0; st < kMmaStages - 1; ++st) {
    if (it.si < seg_end) {
      lay |= (unsigned)load(st, it) << (2 * st);
      advance(it);
    }
    cp_async_commit();
  }
  int buf = 0;
  KIter cit{P.seg0, 0, 0, 0};
  settle(cit);
  while (cit.si < seg_end) {
    cp_async_wait<kMmaStages - 2>();
    __syncthreads();
    {
      const int nb = (buf + kMmaStages - 1) % kMmaStages;
      if (it.si < seg_end) {
        lay = (lay & ~(3u << (2 * nb))) | ((unsigned)load(nb, it) << (2 * nb));
        advance(it);
      }
      cp_async_commit();
    }
    const unsigned l = (lay >> (2 * buf)) & 3u;
    const double *as = smem + buf * SM::STAGE;
    const double *bs = as + SM::A_ELEMS;
    // per-lane fragment addressing: A (m = g, k = t), B (k = t, n = g)
    const int a_line_step = (l & 1) ? SM::LDK : 1;       // next m
    const int a_k_step = (l & 1) ? 1 : SM::LDKM;          // next k
    const int b_line_step = (l & 2) ? SM::LDK : 1;       // next n
    const int b_k_step = (l & 2) ? 1 : SM::LDKN;
    const double *ap = as + (wm0 + g) * a_line_step + t * a_k_step;
    const double *bp = bs + (wn0 + g) * b_line_step + t * b_k_step;
#pragma unroll
    for (int k4 = 0; k4 < BK / 4; ++k4) {
      double a[MT], b[NT];
#pragma unroll
      for (int i = 0; i < MT; ++i) a[i] = ap[(8 * i) * a_line_step + 4 * k4 * a_k_step];
#pragma unroll
      for (int j = 0; j < NT; ++j) b[j] = bp[(8 * j) * b_line_step + 4 * k4 * b_k_step];
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) dmma884(acc[i][j], a[i], b[j]);
    }
    buf = (buf + 1) % kMmaStages;
    advance(cit);
  }
  cp_async_wait<0>();

  double *C = base_ptr(bases, P.cbase) + P.c_off;
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int m = tile.m0 + wm0 + 8 * i + g;
    if (m >= P.M) continue;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int n = tile.n0 + wn0 + 8 * j + 2 * t + h;
        if (n >= P.N) continue;
        double *c = C + m + (long long)n * P.ldc;
        const double v = P.alpha * acc[i][j][h];
        if (P.split > 1)
          atomicAdd(c, v);
        else
          *c = (P.beta == 0.0) ? v : v + P.beta * (*c);
      }
    }
  }
}

// beta pre-pass for problems whose tiles accumulate with atomics
__global__ void gemm_scale_c_kernel(const GemmProb *__restrict__ probs, int nprobs,
                                    GemmBases bases) {
  for (int p = blockIdx.y; p < nprobs; p += gridDim.y) {
    const GemmProb P = probs[p];
    if (P.split <= 1) continue;
    double *C = base_ptr(bases, P.cbase) + P.c_off;
    const long long total = (long long)P.M * P.N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
      const long long m = e % P.M, n = e / P.M;
      double *c = C + m + n * P.ldc;
      *c = (P.beta == 0.0) ? 0.0 : P.beta * (*c);
    }
  }
}

template <int BM, int BN, int WM, int WN>
void launch_gemm(const GemmPlan &plan, const GemmBases &bases, cudaStream_t stream) {
  const int engine = gemm_f64_engine();
  if (engine == 1) {
    static bool configured = false;
    const size_t smem = MmaSmem<BM, BN, 16>::bytes;
    if (!configured) {
      HB_CUDA(cudaFuncSetAttribute(gemm_f64_mma_kernel<BM, BN, WM, WN, 16>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      configured = true;
    }
    gemm_f64_mma_kernel<BM, BN, WM, WN, 16><<<plan.ntiles, kThreads, smem, stream>>>(
        plan.segs, plan.probs, plan.tiles, bases);
    HB_LAUNCHED();
    return;
  }
  if (engine == 2) {
    static bool configured = false;
    const size_t smem = MmaSmem<BM, BN, 32>::bytes;
    if (!configured) {
      HB_CUDA(cudaFuncSetAttribute(gemm_f64_mma_kernel<BM, BN, WM, WN, 32>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      configured = true;
    }
    gemm_f64_mma_kernel<BM, BN, WM, WN, 32><<<plan.ntiles, kThreads, smem, stream>>>(
        plan.segs, plan.probs, plan.tiles, bases);
    HB_LAUNCHED();
    return;
  }
  static bool configured = false;
  const size_t smem = Smem<BM, BN>::bytes;
  if (!configured) {
    HB_CUDA(cudaFuncSetAttribute(gemm_f64_kernel<BM, BN>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = true;
  }
  gemm_f64_kernel<BM, BN><<<plan.ntiles, kThreads, smem, stream>>>(plan.segs, plan.probs,
                                                                   plan.tiles, bases);
  HB_LAUNCHED();
}

}  // namespace

GemmPlan::~GemmPlan() {
  if (!dev) return;
  if (transient)
    cudaFreeAsync(dev, stream);
  else
    cudaFree(dev);
}

void gemm_plan_build(GemmPlan &plan, GemmBatch &batch, TileShape shape, bool allow_split,
                     cudaStream_t stream, bool transient) {
  const auto t_start = std::chrono::steady_clock::now();
  struct Clock {
    std::chrono::steady_clock::time_point t;
    ~Clock() {
      plan_host_ms() +=
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
    }
  } clock{t_start};
  const int BM = tile_rows(shape);
  const int BN = tile_cols(shape);
  plan.shape = shape;
  auto &probs = batch.probs;
  std::vector<long long> ktot(probs.size(), 0);
  long long base_tiles = 0;
  double work = 0.0;
  for (size_t p = 0; p < probs.size(); ++p) {
    for (int s = 0; s < probs[p].nseg; ++s) ktot[p] += batch.segs[probs[p].seg0 + s].K;
    gemm_flops_counter() += 2.0 * probs[p].M * (double)probs[p].N * (double)ktot[p];
    const long long mn =
        (long long)((probs[p].M + BM - 1) / BM) * ((probs[p].N + BN - 1) / BN);
    base_tiles += mn;
    work += (double)mn * (double)std::max<long long>(ktot[p], 1);
  }
  const long long target = 4LL * num_sms();
  // per problem: its K split and the K length of its tiles
  plan.any_split = false;
  std::vector<long long> chunk_of(probs.size(), 0);
  for (size_t p = 0; p < probs.size(); ++p) {
    GemmProb &P = probs[p];
    if (P.M <= 0 || P.N <= 0) continue;
    // Split K so that no tile carries much more than an even share of the
    // batch's work (the longest tile bounds the launch), and to fill the GPU.
    long long split = 1;
    if (allow_split && ktot[p] > 2 * 256) {
      const double per_tile = work / (double)target;          // ideal work per tile
      const double mine = (double)std::max<long long>(ktot[p], 1);
      split = (long long)std::ceil(mine / std::max(per_tile, 512.0));
      split = std::max<long long>(1, std::min<long long>(split, ktot[p] / 256));
    }
    long long chunk = (ktot[p] + split - 1) / split;
    chunk = (chunk + kBK - 1) / kBK * kBK;
    if (chunk <= 0) chunk = kBK;
    split = std::max<long long>(1, (ktot[p] + chunk - 1) / chunk);
    P.split = (int)split;
    if (split > 1) plan.any_split = true;
    chunk_of[p] = split == 1 ? ktot[p] : chunk;
  }
  // tiles of the problems with the longest K ranges first, for load balance
  // (ordering the problems, not the tiles: a problem's tiles share their K
  // length but for a shorter last split)
  std::vector<int> order(probs.size());
  for (size_t p = 0; p < probs.size(); ++p) order[p] = (int)p;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return chunk_of[a] > chunk_of[b]; });
  std::vector<GemmTile> tiles;
  tiles.reserve(base_tiles);
  for (int p : order) {
    const GemmProb &P = probs[p];
    if (P.M <= 0 || P.N <= 0) continue;
    const int mt = (P.M + BM - 1) / BM, nt = (P.N + BN - 1) / BN;
    const long long chunk = chunk_of[p];
    for (int mi = 0; mi < mt; ++mi)
      for (int ni = 0; ni < nt; ++ni)
        for (long long si = 0; si < P.split; ++si) {
          GemmTile t;
          t.prob = p;
          t.m0 = mi * BM;
          t.n0 = ni * BN;
          t.k0 = (int)(si * chunk);
          t.k1 = (int)std::min<long long>(ktot[p], (si + 1) * chunk);
          if (P.split == 1) t.k1 = (int)ktot[p];
          tiles.push_back(t);
        }
  }
  plan.ntiles = (int)tiles.size();
  plan.nprobs = (int)probs.size();
  const size_t bs = batch.segs.size() * sizeof(GemmSeg);
  const size_t bp = probs.size() * sizeof(GemmProb);
  const size_t bt = tiles.size() * sizeof(GemmTile);
  const size_t total = align_up(bs, 256) + align_up(bp, 256) + align_up(bt, 256) + 256;
  if (plan.dev) {
    if (plan.transient)
      cudaFreeAsync(plan.dev, plan.stream);
    else
      cudaFree(plan.dev);
    plan.dev = nullptr;
  }
  plan.transient = transient;
  plan.stream = stream;
  if (transient)
    HB_CUDA(cudaMallocAsync(&plan.dev, total, stream));
  else
    HB_CUDA(cudaMalloc(&plan.dev, total));
  char *base = (char *)plan.dev;
  plan.segs = (GemmSeg *)base;
  plan.probs = (GemmProb *)(base + align_up(bs, 256));
  plan.tiles = (GemmTile *)(base + align_up(bs, 256) + align_up(bp, 256));
  std::unique_ptr<char[]> host(new char[total]);   // padding bytes are never read
  if (bs) std::memcpy(host.get(), batch.segs.data(), bs);
  if (bp) std::memcpy(host.get() + align_up(bs, 256), probs.data(), bp);
  if (bt) std::memcpy(host.get() + align_up(bs, 256) + align_up(bp, 256), tiles.data(), bt);
  // staged through the pinned ring: the host buffer may go away at once, and
  // the host does not wait for the stream
  h2d_async(plan.dev, host.get(), total, stream);
  if (!transient) HB_CUDA(cudaStreamSynchronize(stream));
}

void gemm_plan_run(const GemmPlan &plan, const GemmBases &bases, cudaStream_t stream) {
  if (plan.ntiles == 0) return;
  if (plan.any_split) {
    dim3 grid(64, std::min(plan.nprobs, 1024));
    gemm_scale_c_kernel<<<grid, 256, 0, stream>>>(plan.probs, plan.nprobs, bases);
    HB_LAUNCHED();
  }
  switch (plan.shape) {
    case TileShape::M128N64: launch_gemm<128, 64, 32, 32>(plan, bases, stream); break;
    case TileShape::M64N128: launch_gemm<64, 128, 32, 32>(plan, bases, stream); break;
    case TileShape::M32N128: launch_gemm<32, 128, 32, 16>(plan, bases, stream); break;
    case TileShape::M32N256: launch_gemm<32, 256, 32, 32>(plan, bases, stream); break;
  }
}

void gemm_f64_run(GemmBatch &batch, const GemmBases &bases, TileShape shape, cudaStream_t stream,
                  bool allow_split) {
  if (batch.empty()) return;
  GemmPlan plan;
  gemm_plan_build(plan, batch, shape, allow_split, stream, true);
  gemm_plan_run(plan, bases, stream);
}

}  // namespace hb
