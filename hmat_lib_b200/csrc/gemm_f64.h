// Variable-batched, K-segmented FP64 GEMM engine.
//
// A problem computes C (M x N) = alpha * sum_s op(A_s) op(B_s) + beta * C,
// where the segments s share M and N and each contributes its own K_s; this
// lets one output tile accumulate a leaf product and every level's low-rank
// product in registers (one store per output element).  A problem may be
// split along its concatenated K range into several tiles that add their
// partial sums with FP64 atomics (C is then pre-scaled by beta in a separate
// pass of the same launch sequence).
//
// Every pointer is stored as (base slot, element offset) so that a plan --
// the device copy of the descriptors -- can be reused with new buffers: the
// kernels receive the base addresses as launch arguments.
#pragma once

#include <vector>

#include "common.h"
#include "kernelspec.cuh"

namespace hb {

constexpr int kGemmBases = 6;

// Base addresses of the launch; `gen` defines the operands of base slot
// kGenSlot (kernel-matrix entries computed in the loaders, offset =
// gen_offset(row0, col0) of the block, leading dimension unused).
struct GemmBases {
  double *p[kGemmBases];
  KernelSpec gen;
};

struct GemmSeg {
  long long a_off, b_off;
  long long lda, ldb;
  int K;
  unsigned char ta;     // 0: A is M x K column-major; 1: A stored K x M (op = A^T)
  unsigned char tb;     // 0: B is K x N column-major; 1: B stored N x K (op = B^T)
  unsigned char abase, bbase;
};

struct GemmProb {
  long long c_off;
  long long ldc;
  int M, N;
  int seg0, nseg;
  int cbase;
  int split;            // number of K-split tiles per (m, n) tile (1: plain store)
  double alpha, beta;
};

struct GemmTile {
  int prob;
  int m0, n0;
  int k0, k1;           // range in the problem's concatenated K index
};

// Output tile per CTA.  The 32-row shapes serve skinny problems (a few rows:
// the projections V^T X of low-rank blocks).
enum class TileShape { M128N64 = 0, M64N128 = 1, M32N128 = 2, M32N256 = 3 };
inline int tile_rows(TileShape t) {
  return t == TileShape::M128N64 ? 128 : t == TileShape::M64N128 ? 64 : 32;
}
inline int tile_cols(TileShape t) {
  return t == TileShape::M128N64 ? 64 : t == TileShape::M32N256 ? 256 : 128;
}

struct GemmBatch {
  std::vector<GemmSeg> segs;
  std::vector<GemmProb> probs;

  int add(int cbase, long long c_off, long long ldc, int M, int N, double alpha = 1.0,
          double beta = 0.0) {
    probs.push_back(GemmProb{c_off, ldc, M, N, (int)segs.size(), 0, cbase, 1, alpha, beta});
    return (int)probs.size() - 1;
  }
  // op(A) is M x K, op(B) is K x N.
  void seg(int prob, int abase, long long a_off, long long lda, int ta, int bbase,
           long long b_off, long long ldb, int tb, int K) {
    if (K <= 0) return;
    GemmProb &p = probs[prob];
    HB_REQUIRE(p.nseg == 0 || p.seg0 + p.nseg == (int)segs.size(), INPUT_ERROR,
               "segments of one GEMM problem must be added together");
    if (p.nseg == 0) p.seg0 = (int)segs.size();
    segs.push_back(GemmSeg{a_off, b_off, lda, ldb, K, (unsigned char)ta, (unsigned char)tb,
                           (unsigned char)abase, (unsigned char)bbase});
    p.nseg += 1;
  }
  bool empty() const { return probs.empty(); }
};

// Device-resident plan: descriptors + tile list, reusable across calls that
// use the same geometry with different base buffers.
struct GemmPlan {
  TileShape shape = TileShape::M128N64;
  int ntiles = 0;
  int nprobs = 0;
  bool any_split = false;
  void *dev = nullptr;          // one allocation holding the three arrays
  bool transient = false;       // dev is stream-ordered (freed with cudaFreeAsync on `stream`)
  cudaStream_t stream = nullptr;
  GemmSeg *segs = nullptr;
  GemmProb *probs = nullptr;
  GemmTile *tiles = nullptr;
  GemmPlan() = default;
  GemmPlan(const GemmPlan &) = delete;
  GemmPlan &operator=(const GemmPlan &) = delete;
  ~GemmPlan();
};

// Builds the tile list (splitting long K ranges when the batch would not
// fill the GPU) and uploads it.  A transient plan lives in stream-ordered
// memory of `stream` and is released in stream order: no host
// synchronisation.
void gemm_plan_build(GemmPlan &plan, GemmBatch &batch, TileShape shape, bool allow_split,
                     cudaStream_t stream, bool transient = false);

// Launches a plan: the beta pre-pass for split problems, then the GEMM.
void gemm_plan_run(const GemmPlan &plan, const GemmBases &bases, cudaStream_t stream);

// FP64 multiply-add work (2 M N K per problem) of every GEMM plan built on
// the calling thread since the counter was last reset (build statistics).
double &gemm_flops_counter();
// Host milliseconds spent making GEMM and TSQR plans on this thread (reset by
// the caller).
double &plan_host_ms();

// Which kernel runs the FP64 products (option gemm_f64_engine): 1 the FP64
// tensor-core (DMMA) kernel, 0 the DFMA kernel.
int gemm_f64_engine();

// One-shot convenience: plan, run, release (stream-ordered).
void gemm_f64_run(GemmBatch &batch, const GemmBases &bases, TileShape shape, cudaStream_t stream,
                  bool allow_split = true);

}  // namespace hb
