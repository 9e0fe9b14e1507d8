// Mixed-precision products on the 5th-generation tensor cores: FP64 matrices
// split into int8 slices, products of slices accumulated exactly in int32 by
// tcgen05.mma kind::i8, recombined in FP64.
//
// Splitting (error-free, after Ozaki et al., "Error-free transformations of
// matrix multiplication by using fast routines of matrix multiplication and
// its applications", Numer. Algorithms 2012, with integer slices): each row r
// of A is scaled by 2^-e_r so that |A_rk 2^-e_r| <= 127/128, then written as
// sum_p a^(p) 2^(-7p) with integers a^(1) in [-127, 127] and a^(p) in
// [-64, 64] for p > 1 (round to nearest at every step, so each slice carries
// 7 new bits); columns of B likewise with 2^-f_j.  Then
//   (A B)_rj ~= 2^(e_r + f_j) sum_{t=2}^{S+1} 2^(-7t) sum_{p+q=t} (a^(p) b^(q))_rj
// keeping the S(S+1)/2 slice products with p + q <= S + 1.  Each inner sum is
// one int32 TMEM accumulator.  The largest group (p + q = S + 1) adds at most
// 2*127*64 + 4*64*64 = 32640 per k, so the sums are exact for K <= 65536.
// With S = 6 the truncation error is about 2^-42 relative to
// |A_r|_max |B_j|_max per term.
//
// Operands live in global memory in the blocked layout the MMA reads from
// shared memory, so one K-block of a tile is a single contiguous bulk copy:
// a tile of R lines (rows of A, or columns of B) is a sequence of K-blocks of
// 32 bytes; K-block = [slice 0..S-1][line / 8][k-chunk 0..1][line % 8][16
// bytes of k] (no swizzle, K-major 8 x 16-byte core matrices: 128 bytes
// between k-chunks, 256 bytes between 8-line groups, R * 32 bytes between
// slices).
#pragma once

#include <cstdint>
#include <vector>

#include "common.h"

namespace hb {

constexpr int kOzSlices = 6;                                   // S
constexpr int kOzKBlock = 32;                                  // K bytes per stage (one k-step)
constexpr int kOzRowsA = 128;                                  // A tile lines (MMA M)
constexpr int kOzMaxNw = 64;                                   // widest B tile
constexpr int kOzABlock = kOzSlices * kOzRowsA * kOzKBlock;    // 24576 bytes
constexpr int kOzMaxK = 65536;                                 // exact int32 group sums

__host__ __device__ constexpr int oz_bblock(int nw) { return kOzSlices * nw * kOzKBlock; }

// Byte offset of element (line, k) of slice `p` inside a tile of R lines.
__host__ __device__ inline long long oz_offset(int R, int p, int line, int k) {
  return (long long)(k >> 5) * (kOzSlices * R * kOzKBlock) + (long long)p * R * kOzKBlock +
         (line >> 3) * 256 + ((k >> 4) & 1) * 128 + (line & 7) * 16 + (k & 15);
}

// One K range of a tile: `nkb` K-blocks of A starting at `a` (kOzABlock bytes
// each) against as many K-blocks of B starting at `b` (oz_bblock(nw) each).
struct OzSeg {
  const uint8_t *a;
  const uint8_t *b;
  int nkb;
  int pad_;
};

// One 128 x nw output tile: the K segments seg0 .. seg0 + nseg - 1 all share
// the row exponents rexp[0 .. rows) and column exponents cexp[0 .. cols), so
// the tile is recombined once.  Element (r, j) goes to cbase[c_off + r + j ldc].
// rmax, if set, receives (atomic max, double bits) the largest |result| of
// every row of the tile.
struct OzTile {
  int seg0, nseg;  // at most 32 segments
  int nkb;         // K-blocks of all segments (set by ozaki_schedule)
  int rows, cols;
  int nw;          // B tile width: multiple of 16, <= 64
  int atomic;      // 1: add atomically (K split over several tiles)
  long long c_off, ldc;
  const int *rexp, *cexp;
  unsigned long long *rmax;
};

// Persistent grid for a tile list: one CTA per SM, at most one per tile.
int ozaki_grid(int ntiles);

// Orders `tiles` for a persistent grid of `grid` CTAs and returns where each
// CTA's run of tiles starts (grid + 1 entries; CTA b takes tiles
// [start[b], start[b+1])).  Tiles are assigned longest first to the least
// loaded CTA, a tile's cost being its K-blocks times its width plus a fixed
// per-tile cost (the accumulator hand-over), so that CTAs finish together.
// Option ozaki_schedule = 0 gives tile i to CTA i mod grid instead.
std::vector<int> ozaki_schedule(std::vector<OzTile> &tiles, const std::vector<OzSeg> &segs,
                                int grid);

// Runs all tiles with the persistent grid of a schedule.  `status` (device
// int) is set to 1 if a bounded barrier wait ran out.
void ozaki_gemm(const OzSeg *d_segs, const OzTile *d_tiles, const int *d_starts, int grid,
                double *cbase, int *d_status, cudaStream_t stream);

// Largest |value| per line of a strided FP64 matrix, element (line, k) at
// src[line * s_line + k * s_k], combined by atomic max into out[line] (the
// bit pattern of a non-negative double; zero it first).  A NULL src stands
// for the `xbase` argument of the launch.  item0: prefix over the jobs of
// their work items (filled when the batch is made).
struct MaxJob {
  const double *src;
  long long s_line, s_k;
  int lines, K;
  unsigned long long *out;
  long long item0;
};

// Scales every line by its exponent (from maxabs[line]) and writes the int8
// slices in the blocked layout: lines [0, ntiles R) (zero past `lines`),
// K-blocks [kb0, kb0 + nkb) of each tile (zero past K).  exp_out, if set,
// receives the exponent of every line.
struct SliceJob {
  const double *src;
  long long s_line, s_k;
  int lines, K;
  int R, ntiles, kb0, nkb;
  uint8_t *dst;
  long long tile_stride;
  const unsigned long long *maxabs;
  int *exp_out;
  long long item0;
};

// Job lists uploaded once.  A slice batch is either all K-contiguous (s_k = 1:
// read through a shared-memory transpose) or all line-contiguous.
struct MaxBatch {
  MaxJob *d = nullptr;
  int n = 0;
  long long items = 0;
};
struct SliceBatch {
  SliceJob *d = nullptr;
  int n = 0;
  long long items = 0;
  bool kcontig = false;
};
// Zero (src NULL) or copy `words` 8-byte words per range, all ranges in one
// launch.
struct CopyRange {
  void *dst;
  const void *src;
  long long words;
};
void ozaki_ranges(const CopyRange *d_ranges, int n, cudaStream_t stream);

MaxBatch ozaki_max_batch(std::vector<MaxJob> jobs, cudaStream_t stream);
SliceBatch ozaki_slice_batch(std::vector<SliceJob> jobs, cudaStream_t stream);
void ozaki_max(const MaxBatch &b, const double *xbase, cudaStream_t stream);
void ozaki_slice(const SliceBatch &b, const double *xbase, cudaStream_t stream);

}  // namespace hb
