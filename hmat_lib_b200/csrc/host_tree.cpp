// Host-side tree skeleton: allocation, linking and freeing of the node
// structs of include/hmat_lib/hodlr.h, plus extraction of the block geometry
// the device engine works from.
//
// Entry points replace hmat_lib src/allocators.c (allocate_tree :229,
// allocate_tree_monolithic :404, compute_construct_tree_array_sizes :499,
// construct_tree :561, free_tree_data :659, free_tree_hodlr :747) and
// src/utils.c:5 (get_highest_s).  Node numbering here is this library's own
// (breadth-first); callers only ever follow the pointers.
#include <cstdlib>
#include <cstring>
#include <new>

#include "host_tree.h"

namespace hb {

HostAllocator &host_allocator() {
  static HostAllocator a{&std::malloc, &std::free};
  return a;
}

void *host_malloc(size_t bytes) { return host_allocator().alloc(bytes ? bytes : 1); }
void host_free(void *p) { if (p) host_allocator().release(p); }

HODLRInternalNode *node_at(HODLRInternalNode *root, int d, int j) {
  HODLRInternalNode *node = root;
  for (int level = d - 1; level >= 0; --level) {
    const int bit = (j >> level) & 1;
    node = node->children[bit ? 3 : 0].internal;
  }
  return node;
}

HODLRLeafNode *diag_leaf(HODLRInternalNode *root, int height, int i) {
  HODLRInternalNode *parent = node_at(root, height - 1, i >> 1);
  return parent->children[(i & 1) ? 3 : 0].leaf;
}

static void init_offdiag(HODLRLeafNode *leaf, HODLRInternalNode *parent) {
  leaf->type = OFFDIAGONAL;
  leaf->parent = parent;
  leaf->data.off_diagonal.u = nullptr;
  leaf->data.off_diagonal.v = nullptr;
  leaf->data.off_diagonal.m = 0;
  leaf->data.off_diagonal.s = 0;
  leaf->data.off_diagonal.n = 0;
}

static void init_diag(HODLRLeafNode *leaf, HODLRInternalNode *parent) {
  leaf->type = DIAGONAL;
  leaf->parent = parent;
  leaf->data.diagonal.data = nullptr;
  leaf->data.diagonal.m = 0;
}

static void init_internal(HODLRInternalNode *node, HODLRInternalNode *parent) {
  for (auto &c : node->children) c.internal = nullptr;
  node->parent = parent;
  node->m = 0;
}

// Links `internal` (2^h - 1 nodes, breadth-first) and `leaves` (off-diagonal
// leaves of node k at 2k, 2k+1; the 2^h diagonal leaves after them).
static void link_tree(int h, TreeHODLR *t, HODLRInternalNode *internal, HODLRLeafNode *leaves,
                      HODLRInternalNode **work_queue, HODLRLeafNode **innermost) {
  const long n_internal = (1L << h) - 1;
  for (long k = 0; k < n_internal; ++k) {
    HODLRInternalNode *parent = k == 0 ? nullptr : &internal[(k - 1) / 2];
    init_internal(&internal[k], parent);
  }
  for (long k = 0; k < n_internal; ++k) {
    HODLRInternalNode *node = &internal[k];
    init_offdiag(&leaves[2 * k], node);
    init_offdiag(&leaves[2 * k + 1], node);
    node->children[1].leaf = &leaves[2 * k];
    node->children[2].leaf = &leaves[2 * k + 1];
    const long left = 2 * k + 1;
    if (left < n_internal) {
      node->children[0].internal = &internal[left];
      node->children[3].internal = &internal[left + 1];
    }
  }
  const long first_bottom = (1L << (h - 1)) - 1;
  const long n_bottom = 1L << (h - 1);
  HODLRLeafNode *diag = leaves + 2 * n_internal;
  for (long i = 0; i < n_bottom; ++i) {
    HODLRInternalNode *node = &internal[first_bottom + i];
    init_diag(&diag[2 * i], node);
    init_diag(&diag[2 * i + 1], node);
    node->children[0].leaf = &diag[2 * i];
    node->children[3].leaf = &diag[2 * i + 1];
    innermost[2 * i] = &diag[2 * i];
    innermost[2 * i + 1] = &diag[2 * i + 1];
    work_queue[i] = node;
  }
  t->height = h;
  t->root = &internal[0];
  t->innermost_leaves = innermost;
  t->len_work_queue = n_bottom;
  t->work_queue = work_queue;
}

// Walk every data pointer of a full tree.
template <class F>
static void for_each_leaf(TreeHODLR *t, F &&f) {
  const int h = t->height;
  for (int d = 0; d < h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      HODLRInternalNode *node = node_at(t->root, d, j);
      f(node->children[1].leaf);
      f(node->children[2].leaf);
    }
  for (long i = 0; i < (1L << h); ++i) f(t->innermost_leaves[i]);
}

// Geometry ------------------------------------------------------------------

Geometry geometry_of_subtree(const HODLRInternalNode *root_c, int height) {
  HB_REQUIRE(root_c != nullptr && height >= 1, INPUT_ERROR, "empty subtree");
  auto *root = const_cast<HODLRInternalNode *>(root_c);
  Geometry g;
  g.h = height;
  const int nleaf = 1 << height;
  g.leaf_m.resize(nleaf);
  g.leaf_off.resize(nleaf + 1);
  g.leaf_off[0] = 0;
  for (int i = 0; i < nleaf; ++i) {
    HODLRLeafNode *leaf = diag_leaf(root, height, i);
    HB_REQUIRE(leaf != nullptr, INPUT_ERROR, "missing diagonal leaf");
    g.leaf_m[i] = leaf->data.diagonal.m;
    HB_REQUIRE(g.leaf_m[i] >= 0, INPUT_ERROR, "negative leaf size");
    g.leaf_off[i + 1] = g.leaf_off[i] + (long long)g.leaf_m[i];
  }
  g.n = (int)g.leaf_off[nleaf];
  g.blocks.resize(2 * (nleaf - 1));
  for (int d = 0; d < height; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      HODLRInternalNode *node = node_at(root, d, j);
      const int span = 1 << (height - d);
      const long long o = g.leaf_off[j * span];
      const long long mid = g.leaf_off[j * span + span / 2];
      const long long end = g.leaf_off[(j + 1) * span];
      for (int c = 1; c <= 2; ++c) {
        const NodeOffDiagonal &od = node->children[c].leaf->data.off_diagonal;
        BlockDesc &b = g.blocks[block_index(d, j, c)];
        b.depth = d;
        if (c == 1) {
          b.r0 = (int)o; b.c0 = (int)mid;
          b.m = (int)(mid - o); b.n = (int)(end - mid);
        } else {
          b.r0 = (int)mid; b.c0 = (int)o;
          b.m = (int)(end - mid); b.n = (int)(mid - o);
        }
        HB_REQUIRE(od.m == b.m && od.n == b.n, INPUT_ERROR,
                   "off-diagonal block sizes disagree with the diagonal leaves");
        HB_REQUIRE(od.s >= 0, INPUT_ERROR, "negative rank");
        b.s = od.s;
        b.u_off = b.v_off = 0;
      }
    }
  return g;
}

Geometry geometry_of(const TreeHODLR *t) {
  HB_REQUIRE(t != nullptr && t->root != nullptr, INPUT_ERROR, "NULL tree");
  return geometry_of_subtree(t->root, t->height);
}

Geometry geometry_from_leaves(int h, const std::vector<int> &leaf) {
  Geometry g;
  g.h = h;
  g.leaf_m = leaf;
  g.leaf_off.assign(leaf.size() + 1, 0);
  for (size_t i = 0; i < leaf.size(); ++i) g.leaf_off[i + 1] = g.leaf_off[i] + leaf[i];
  g.n = (int)g.leaf_off.back();
  g.blocks.resize(g.nblock());
  for (int d = 0; d < h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      const int span = 1 << (h - d);
      const long long o = g.leaf_off[j * span], mid = g.leaf_off[j * span + span / 2],
                      end = g.leaf_off[(j + 1) * span];
      g.blocks[block_index(d, j, 1)] =
          BlockDesc{(int)o, (int)mid, (int)(mid - o), (int)(end - mid), 0, d, 0, 0};
      g.blocks[block_index(d, j, 2)] =
          BlockDesc{(int)mid, (int)o, (int)(end - mid), (int)(mid - o), 0, d, 0, 0};
    }
  return g;
}

}  // namespace hb

using namespace hb;

extern "C" {

void compute_construct_tree_array_sizes(const int height, size_t *size_internal_nodes,
                                        size_t *size_leaf_nodes, size_t *size_work_queue,
                                        size_t *size_innermost_leaves) {
  const size_t bottom = (size_t)1 << (height - 1);
  *size_work_queue = bottom * sizeof(HODLRInternalNode *);
  *size_internal_nodes = (2 * bottom - 1) * sizeof(HODLRInternalNode);
  *size_innermost_leaves = 2 * bottom * sizeof(HODLRLeafNode *);
  *size_leaf_nodes = (6 * bottom - 2) * sizeof(HODLRLeafNode);
}

void construct_tree(const int height, TreeHODLR *hodlr, HODLRInternalNode *internal_nodes,
                    HODLRLeafNode *leaf_nodes, HODLRInternalNode **work_queue,
                    HODLRLeafNode **innermost_leaves, int *ierr) {
  if (height < 1) {
    *ierr = INPUT_ERROR;
    return;
  }
  link_tree(height, hodlr, internal_nodes, leaf_nodes, work_queue, innermost_leaves);
  hodlr->memory_internal_ptr = internal_nodes;
  hodlr->memory_leaf_ptr = leaf_nodes;
  *ierr = SUCCESS;
}

TreeHODLR *allocate_tree_monolithic(const int height, int *ierr) {
  if (height < 1 || height > 30) {
    *ierr = INPUT_ERROR;
    return nullptr;
  }
  size_t si, sl, sq, sil;
  compute_construct_tree_array_sizes(height, &si, &sl, &sq, &sil);
  auto *t = (TreeHODLR *)host_malloc(sizeof(TreeHODLR));
  auto *internal = (HODLRInternalNode *)host_malloc(si);
  auto *leaves = (HODLRLeafNode *)host_malloc(sl);
  auto *queue = (HODLRInternalNode **)host_malloc(sq);
  auto *innermost = (HODLRLeafNode **)host_malloc(sil);
  if (!t || !internal || !leaves || !queue || !innermost) {
    host_free(t); host_free(internal); host_free(leaves); host_free(queue); host_free(innermost);
    *ierr = ALLOCATION_FAILURE;
    return nullptr;
  }
  construct_tree(height, t, internal, leaves, queue, innermost, ierr);
  return t;
}

// Piecewise variant: every node in its own allocation, as hmat_lib's
// allocate_tree does; memory_*_ptr stay NULL so free_tree_hodlr frees the
// nodes one by one.
TreeHODLR *allocate_tree(const int height, int *ierr) {
  if (height < 1 || height > 30) {
    *ierr = INPUT_ERROR;
    return nullptr;
  }
  const long n_internal = (1L << height) - 1;
  const long n_bottom = 1L << (height - 1);
  auto *t = (TreeHODLR *)host_malloc(sizeof(TreeHODLR));
  auto *queue = (HODLRInternalNode **)host_malloc(n_bottom * sizeof(HODLRInternalNode *));
  auto *innermost = (HODLRLeafNode **)host_malloc(2 * n_bottom * sizeof(HODLRLeafNode *));
  std::vector<HODLRInternalNode *> nodes(n_internal, nullptr);
  std::vector<HODLRLeafNode *> leaves(2 * n_internal + 2 * n_bottom, nullptr);
  bool ok = t && queue && innermost;
  for (auto &p : nodes)
    if (ok && !(p = (HODLRInternalNode *)host_malloc(sizeof(HODLRInternalNode)))) ok = false;
  for (auto &p : leaves)
    if (ok && !(p = (HODLRLeafNode *)host_malloc(sizeof(HODLRLeafNode)))) ok = false;
  if (!ok) {
    for (auto *p : nodes) host_free(p);
    for (auto *p : leaves) host_free(p);
    host_free(t); host_free(queue); host_free(innermost);
    *ierr = ALLOCATION_FAILURE;
    return nullptr;
  }
  for (long k = 0; k < n_internal; ++k) init_internal(nodes[k], k ? nodes[(k - 1) / 2] : nullptr);
  for (long k = 0; k < n_internal; ++k) {
    init_offdiag(leaves[2 * k], nodes[k]);
    init_offdiag(leaves[2 * k + 1], nodes[k]);
    nodes[k]->children[1].leaf = leaves[2 * k];
    nodes[k]->children[2].leaf = leaves[2 * k + 1];
    if (2 * k + 1 < n_internal) {
      nodes[k]->children[0].internal = nodes[2 * k + 1];
      nodes[k]->children[3].internal = nodes[2 * k + 2];
    }
  }
  for (long i = 0; i < n_bottom; ++i) {
    HODLRInternalNode *node = nodes[n_bottom - 1 + i];
    HODLRLeafNode *a = leaves[2 * n_internal + 2 * i], *b = leaves[2 * n_internal + 2 * i + 1];
    init_diag(a, node);
    init_diag(b, node);
    node->children[0].leaf = a;
    node->children[3].leaf = b;
    innermost[2 * i] = a;
    innermost[2 * i + 1] = b;
    queue[i] = node;
  }
  t->height = height;
  t->root = nodes[0];
  t->innermost_leaves = innermost;
  t->len_work_queue = n_bottom;
  t->work_queue = queue;
  t->memory_internal_ptr = nullptr;
  t->memory_leaf_ptr = nullptr;
  *ierr = SUCCESS;
  return t;
}

void free_tree_data(TreeHODLR *hodlr) {
  if (hodlr == nullptr || hodlr->root == nullptr) return;
  forget_device_tree(hodlr);
  for_each_leaf(hodlr, [](HODLRLeafNode *leaf) {
    if (leaf == nullptr) return;
    if (leaf->type == DIAGONAL) {
      host_free(leaf->data.diagonal.data);
      leaf->data.diagonal.data = nullptr;
    } else {
      host_free(leaf->data.off_diagonal.u);
      host_free(leaf->data.off_diagonal.v);
      leaf->data.off_diagonal.u = nullptr;
      leaf->data.off_diagonal.v = nullptr;
    }
  });
}

void free_tree_hodlr(TreeHODLR **hodlr_ptr) {
  if (hodlr_ptr == nullptr || *hodlr_ptr == nullptr) return;
  TreeHODLR *t = *hodlr_ptr;
  free_tree_data(t);
  if (t->memory_leaf_ptr != nullptr) {
    host_free(t->memory_leaf_ptr);
    host_free(t->memory_internal_ptr);
  } else if (t->root != nullptr) {
    const int h = t->height;
    for (int d = h - 1; d >= 0; --d)
      for (int j = 0; j < (1 << d); ++j) {
        HODLRInternalNode *node = node_at(t->root, d, j);
        host_free(node->children[1].leaf);
        host_free(node->children[2].leaf);
        if (d == h - 1) {
          host_free(node->children[0].leaf);
          host_free(node->children[3].leaf);
        }
      }
    // internal nodes last, deepest first (node_at needs the upper ones)
    for (int d = h - 1; d >= 0; --d)
      for (int j = 0; j < (1 << d); ++j) host_free(node_at(t->root, d, j));
  }
  host_free(t->work_queue);
  host_free(t->innermost_leaves);
  host_free(t);
  *hodlr_ptr = nullptr;
}

int get_highest_s(const TreeHODLR *const hodlr) {
  if (hodlr == nullptr || hodlr->root == nullptr) return 0;
  int best = 0;
  for (int d = 0; d < hodlr->height; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      HODLRInternalNode *node = node_at(hodlr->root, d, j);
      for (int c = 1; c <= 2; ++c) {
        const int s = node->children[c].leaf->data.off_diagonal.s;
        if (s > best) best = s;
      }
    }
  return best;
}

}  // extern "C"
