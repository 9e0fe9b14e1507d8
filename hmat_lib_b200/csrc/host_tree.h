// Host tree helpers shared by the C-ABI layer.
#pragma once

#include <cstddef>
#include <vector>

#include "../../include/hmat_lib/hodlr.h"
#include "../../include/hmat_lib/allocators.h"
#include "common.h"

namespace hb {

// Allocator used for every host allocation the library makes on behalf of a
// caller (tree nodes, factor copies, malloc'd results).  Replaceable through
// hodlr_b200_set_host_allocator so tests can inject allocation failures.
struct HostAllocator {
  void *(*alloc)(size_t);
  void (*release)(void *);
};
HostAllocator &host_allocator();
void *host_malloc(size_t bytes);
void host_free(void *p);

// Block geometry of a (sub)tree, derived from its leaf sizes; offsets are
// relative to the (sub)tree's first row.
struct Geometry {
  int h = 0;
  int n = 0;
  std::vector<int> leaf_m;
  std::vector<long long> leaf_off;   // 2^h + 1 prefix sums
  std::vector<BlockDesc> blocks;     // indexed by block_index(d, j, c)

  int nleaf() const { return 1 << h; }
  int nblock() const { return 2 * ((1 << h) - 1); }
  int max_rank() const {
    int s = 0;
    for (auto &b : blocks) s = b.s > s ? b.s : s;
    return s;
  }
};

HODLRInternalNode *node_at(HODLRInternalNode *root, int d, int j);
HODLRLeafNode *diag_leaf(HODLRInternalNode *root, int height, int i);

Geometry geometry_of(const TreeHODLR *t);
// Geometry of a tree of height h with the given 2^h leaf sizes (ranks 0): the
// block of child 1 of node (d, j) spans the node's first half of rows and its
// second half of columns, child 2 the reverse.
Geometry geometry_from_leaves(int h, const std::vector<int> &leaf);
Geometry geometry_of_subtree(const HODLRInternalNode *root, int height);

// Drop any device copy registered for this host tree (dtree.cu).
void forget_device_tree(const TreeHODLR *t);

}  // namespace hb
