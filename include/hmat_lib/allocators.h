/* Tree skeleton allocation.  Same entry points as hmat_lib
 * include/hmat_lib/allocators.h:5-49 (production ABI, i.e. without the
 * _TEST_HODLR allocator-injection parameters). */
#pragma once

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

struct TreeHODLR;
struct HODLRInternalNode;
struct HODLRLeafNode;

/* One malloc per node (hmat_lib src/allocators.c:229). */
struct TreeHODLR *allocate_tree(const int height, int *ierr);

/* Four block allocations, nodes contiguous (hmat_lib src/allocators.c:404). */
struct TreeHODLR *allocate_tree_monolithic(const int height, int *ierr);

/* Frees data and skeleton; sets *hodlr_ptr to NULL
 * (hmat_lib src/allocators.c:747). */
void free_tree_hodlr(struct TreeHODLR **hodlr_ptr);

/* Frees only the leaf data and sets the data pointers to NULL
 * (hmat_lib src/allocators.c:659). */
void free_tree_data(struct TreeHODLR *hodlr);

/* Byte sizes of the four arrays construct_tree links together
 * (hmat_lib src/allocators.c:499). */
void compute_construct_tree_array_sizes(
  const int height,
  size_t *size_internal_nodes,
  size_t *size_leaf_nodes,
  size_t *size_work_queue,
  size_t *size_innermost_leaves
);

/* Links caller-provided node arrays into a tree
 * (hmat_lib src/allocators.c:561). */
void construct_tree(
  const int height,
  struct TreeHODLR *hodlr,
  struct HODLRInternalNode *internal_nodes,
  struct HODLRLeafNode *leaf_nodes,
  struct HODLRInternalNode **work_queue,
  struct HODLRLeafNode **innermost_leaves,
  int *ierr
);

#ifdef __cplusplus
}
#endif
