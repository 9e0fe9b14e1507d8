// Shared definitions of libhodlr_b200: status handling, launch accounting,
// device descriptors of the tree arena.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/hmat_lib/error.h"

namespace hb {

// Error carried from deep inside the engine to the C-ABI boundary, where it
// becomes an hmat_lib ErrorCode plus a message (hodlr_b200_last_error()).
struct Error {
  int code;
  std::string msg;
};

// Host -> device copy of `bytes` from pageable memory that returns without
// waiting for `stream`: the bytes go through a pinned staging ring of the
// calling thread (64 MiB per device, slots recycled once their copy has
// completed); `src` may be reused at once.  A copy from pageable memory would
// make the host wait until the stream reaches it, so a build that uploads
// launch descriptors between launches would run host and GPU in turn.
// Copies larger than half the ring, or into a capturing stream, are plain
// cudaMemcpyAsync calls.
void h2d_async(void *dst, const void *src, size_t bytes, cudaStream_t stream);

void set_last_error(const std::string &msg);
// Records a message that is a string literal, without allocating.
void set_last_error_static(const char *msg);
const char *last_error();

// A failed runtime call also becomes the thread's "last error"; it is read
// back here so that a later launch check does not report it a second time.
#define HB_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      (void)cudaGetLastError();                                              \
      throw ::hb::Error{ALLOCATION_FAILURE,                                  \
                        std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    }                                                                        \
  } while (0)

#define HB_REQUIRE(cond, code, text)                 \
  do {                                               \
    if (!(cond)) throw ::hb::Error{(code), (text)};  \
  } while (0)

// Count of kernels this library launched (reported by the benchmark as its
// own GPU launches).
void count_launch(long long n = 1);
long long launches();

// After every launch: surface configuration errors immediately.
#define HB_LAUNCHED()                                                        \
  do {                                                                       \
    ::hb::count_launch();                                                    \
    cudaError_t e_ = cudaGetLastError();                                     \
    if (e_ != cudaSuccess)                                                   \
      throw ::hb::Error{ALLOCATION_FAILURE,                                  \
                        std::string("kernel launch: ") + cudaGetErrorString(e_)}; \
  } while (0)

int num_sms();

// Runtime knobs (hodlr_b200_set_option).
double option(const char *name, double dflt);
void set_option(const std::string &name, double value);

// ---------------------------------------------------------------------------
// Device-side descriptors of one HODLR stored in an arena of doubles.
//
// Off-diagonal block index: b = 2 * (2^d - 1 + j) + (c - 1) for internal node
// (d, j) and child c (1 top-right, 2 bottom-left).  Leaf i is the i-th
// diagonal block from the top-left.
struct LeafDesc {
  int r0;          // first row/column of the leaf
  int m;           // leaf size
  long long off;   // arena offset of the m x m column-major block
};

struct BlockDesc {
  int r0, c0;      // first row / column of the block in the full matrix
  int m, n, s;     // rows, columns, rank
  int depth;
  long long u_off; // arena offset of U (m x s, ld m)
  long long v_off; // arena offset of V (n x s, ld n)
};

inline int block_index(int d, int j, int c) { return 2 * ((1 << d) - 1 + j) + (c - 1); }

// Rounded-up arena allocation granule (doubles): 32 doubles = 256 bytes keeps
// every factor 256-byte aligned for vectorised and bulk copies.
constexpr long long kArenaAlign = 32;
inline long long align_up(long long x, long long a = kArenaAlign) { return (x + a - 1) / a * a; }

}  // namespace hb
