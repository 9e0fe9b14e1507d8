/*
 * HODLR tree data model of the hodlr-b200 engine.
 *
 * The layout of every struct and enum below is byte-identical to hmat_lib's
 * public data model (hmat_lib include/hmat_lib/hodlr.h:7-263) so that C code
 * written against hmat_lib, which walks the tree directly
 * (root->children[1].leaf->data.off_diagonal.u and so on), compiles and runs
 * unchanged against libhodlr_b200.so.
 *
 * Conventions (all matrices column-major, FP64):
 *   - a diagonal leaf holds a dense m x m block;
 *   - an off-diagonal leaf holds U (m x s), already multiplied by the kept
 *     singular values, and V (n x s) -- V itself, not its transpose;
 *   - an internal node splits its block 2x2: children[0] top-left diagonal,
 *     children[1] top-right off-diagonal, children[2] bottom-left
 *     off-diagonal, children[3] bottom-right diagonal.
 */
#pragma once

enum NodeType {
  DIAGONAL,
  OFFDIAGONAL,
  INTERNAL
};

/* Dense diagonal leaf: `data` is an m x m column-major block. */
struct NodeDiagonal {
  double *data;
  int m;
};

/* Low-rank off-diagonal leaf: block = u * v^T, u is m x s (scaled by the
 * singular values, columns in descending singular-value order), v is n x s. */
struct NodeOffDiagonal {
  double *u;
  double *v;
  int m;
  int s;
  int n;
};

union HODLRData {
  struct NodeDiagonal diagonal;
  struct NodeOffDiagonal off_diagonal;
};

struct HODLRLeafNode {
  enum NodeType type;
  union HODLRData data;
  struct HODLRInternalNode *parent;
};

union HODLRNode {
  struct HODLRLeafNode *leaf;
  struct HODLRInternalNode *internal;
};

struct HODLRInternalNode {
  /* 0: top-left, 1: top-right (leaf), 2: bottom-left (leaf), 3: bottom-right */
  union HODLRNode children[4];
  struct HODLRInternalNode *parent;   /* NULL at the root */
  int m;                              /* size of the block this node covers */
};

struct TreeHODLR {
  int height;                               /* number of splits */
  struct HODLRInternalNode *root;
  struct HODLRLeafNode **innermost_leaves;  /* 2^height diagonal leaves,
                                               top-left to bottom-right */
  long len_work_queue;                      /* 2^(height-1) */
  struct HODLRInternalNode **work_queue;    /* scratch; may change even
                                               through a const tree */
  struct HODLRInternalNode *memory_internal_ptr;  /* non-NULL when the nodes */
  struct HODLRLeafNode *memory_leaf_ptr;          /* were allocated in blocks */
};
