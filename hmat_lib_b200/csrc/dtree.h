// Device-resident HODLR: one arena of doubles holding every diagonal leaf and
// every U / V factor, plus descriptor arrays, and a registry that pairs a host
// TreeHODLR with its device copy.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "gemm_f64.h"
#include "host_tree.h"

namespace hb {

struct ProductPlan;
struct MixedState;

// A captured launch sequence of one product (CUDA graph), replayed by later
// calls with the same tree, op, sizes, buffers and stream.
struct ProductGraph {
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;     // kernels in the graph (for the launch counter)
  ~ProductGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

struct DeviceTree {
  int device = 0;
  Geometry g;                       // blocks carry u_off / v_off into `arena`
  std::vector<LeafDesc> leaves;     // host copy of d_leaves
  double *arena = nullptr;
  long long arena_elems = 0;
  LeafDesc *d_leaves = nullptr;
  BlockDesc *d_blocks = nullptr;
  uint64_t fingerprint = 0;         // of the host tree this mirrors (0: none)
  std::map<std::tuple<int, int, long long, long long, int, int>, std::unique_ptr<ProductPlan>> plans;
  // (op, k, ldx, ldy, min_depth, X, Y, stream) -> graph; an entry holding
  // nullptr marks a signature seen once (captured on its second call)
  std::map<std::tuple<int, int, long long, long long, int, const void *, void *, void *>,
           std::unique_ptr<ProductGraph>>
      graphs;
  std::mutex plan_mutex;
  std::shared_ptr<MixedState> mixed;   // int8 slices of the factors (mixed precision)
  std::shared_ptr<DeviceTree> transposed;   // H^T with the same geometry (mixed op T / L)
  int *mv_woff = nullptr;              // single-vector product: W offset of every block
  double *mv_w = nullptr;              // and W (made on the first such product)

  DeviceTree() = default;
  DeviceTree(const DeviceTree &) = delete;
  DeviceTree &operator=(const DeviceTree &) = delete;
  ~DeviceTree();

  long long storage() const;        // stored doubles (leaves + factors)
};

// Lays out the arena for geometry `g` (ranks included), allocates it and
// uploads the descriptors.  Contents are uninitialised.
std::unique_ptr<DeviceTree> dtree_create(const Geometry &g, cudaStream_t stream);

// Copies every leaf and factor of a host (sub)tree into the arena.
void dtree_upload(DeviceTree &t, HODLRInternalNode *root, cudaStream_t stream);

// Allocates host buffers (library allocator) for every leaf / factor of the
// host tree, copies the arena into them and sets sizes, ranks and pointers.
void dtree_download(const DeviceTree &t, TreeHODLR *host, cudaStream_t stream);

// Fingerprint of a host tree: structure, data pointers and sampled values.
uint64_t host_fingerprint(const TreeHODLR *t);

// Registry ------------------------------------------------------------------
std::shared_ptr<DeviceTree> device_tree_for(const TreeHODLR *t, cudaStream_t stream);
void register_device_tree(const TreeHODLR *t, std::shared_ptr<DeviceTree> dt);

// Library stream of the current device (non-blocking, created on first use).
cudaStream_t lib_stream();

// Stream-ordered scratch allocation.
// Keeps freed stream-ordered memory mapped in the current device's default
// pool (once per device; option pool_keep).
void keep_pool_memory();
double *dev_alloc(size_t elems, cudaStream_t stream);
void dev_free(void *p, cudaStream_t stream);


}  // namespace hb

// The opaque handle of include/hmat_lib/hodlr_b200.h.
struct hodlr_b200_tree_s {
  std::shared_ptr<hb::DeviceTree> p;
};
