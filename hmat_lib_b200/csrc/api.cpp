// C-ABI entry points of libhodlr_b200.so.
//
// The hmat_lib functions keep their signatures, argument meaning, ownership
// rules and error behaviour (include/hmat_lib/*.h); the arithmetic runs on
// the GPU.  Every failure is reported through *ierr (and the message through
// hodlr_b200_last_error()); nothing falls back to the CPU.
#include <cstring>
#include <memory>

#include "../../include/hmat_lib/constructors.h"
#include "../../include/hmat_lib/dense_algebra.h"
#include "../../include/hmat_lib/hodlr_algebra.h"
#include "../../include/hmat_lib/hodlr_b200.h"
#include "../../include/hmat_lib/utils.h"
#include "../../include/hmat_lib/vector_algebra.h"
#include "build.h"
#include "hxh.h"
#include "products.h"
#include "rank_mlp.h"
#include "solve.h"

using namespace hb;

namespace {

int fail(int *ierr, const Error &e) {
  set_last_error(e.msg);
  if (ierr) *ierr = e.code;
  return e.code;
}

// NULL selects the CUDA default stream, as CUDA libraries do.
cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

// Leaf sizes of a tree of height h over m rows with halving splits, the
// top-left child taking m - m/2 (hmat_lib src/constructors.c:60-64).
std::vector<int> halves(int m, int h) {
  std::vector<int> sizes{m};
  for (int l = 0; l < h; ++l) {
    std::vector<int> nxt;
    for (int s : sizes) {
      nxt.push_back(s - s / 2);
      nxt.push_back(s / 2);
    }
    sizes.swap(nxt);
  }
  return sizes;
}

// Writes every node size of the host tree from its leaf sizes, as hmat_lib's
// block sizing does (src/constructors.c:44-176).
void apply_sizes(TreeHODLR *t, const std::vector<int> &leaf) {
  const int h = t->height;
  std::vector<long long> off(leaf.size() + 1, 0);
  for (size_t i = 0; i < leaf.size(); ++i) off[i + 1] = off[i] + leaf[i];
  for (int i = 0; i < (1 << h); ++i) diag_leaf(t->root, h, i)->data.diagonal.m = leaf[i];
  for (int d = 0; d < h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      HODLRInternalNode *node = node_at(t->root, d, j);
      const int span = 1 << (h - d);
      const int a = (int)(off[j * span + span / 2] - off[j * span]);
      const int b = (int)(off[(j + 1) * span] - off[j * span + span / 2]);
      node->m = a + b;
      node->children[1].leaf->data.off_diagonal.m = a;
      node->children[1].leaf->data.off_diagonal.n = b;
      node->children[2].leaf->data.off_diagonal.m = b;
      node->children[2].leaf->data.off_diagonal.n = a;
    }
}

struct DevBuf {
  double *p = nullptr;
  cudaStream_t s;
  explicit DevBuf(size_t elems, cudaStream_t st) : s(st) { p = dev_alloc(elems, st); }
  ~DevBuf() { dev_free(p, s); }
};

// Host matrix (rows x cols, ld) -> packed device buffer (ld = rows).
void h2d(double *dst, const double *src, long long rows, long long cols, long long ld,
         cudaStream_t s) {
  if (rows * cols == 0) return;
  HB_CUDA(cudaMemcpy2DAsync(dst, rows * sizeof(double), src, ld * sizeof(double),
                            rows * sizeof(double), cols, cudaMemcpyHostToDevice, s));
}
void d2h(double *dst, long long ld, const double *src, long long rows, long long cols,
         cudaStream_t s) {
  if (rows * cols == 0) return;
  HB_CUDA(cudaMemcpy2DAsync(dst, ld * sizeof(double), src, rows * sizeof(double),
                            rows * sizeof(double), cols, cudaMemcpyDeviceToHost, s));
}

// Copy streams of the host-buffer products (0: host to device, 1: device to
// host), one pair per device and thread like the library stream.
cudaStream_t copy_stream(int which) {
  static thread_local std::map<std::pair<int, int>, cudaStream_t> streams;
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_pair(dev, which);
  auto it = streams.find(key);
  if (it != streams.end()) return it->second;
  cudaStream_t st;
  HB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  streams[key] = st;
  return st;
}

struct Events {
  std::vector<cudaEvent_t> e;
  explicit Events(size_t n) : e(n, nullptr) {
    for (auto &ev : e) HB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  ~Events() {
    for (auto ev : e)
      if (ev) cudaEventDestroy(ev);
  }
};

// Host-buffer product shared by multiply_vector / multiply_*_dense.
// X is xr x xc (ld ldx); Y has the same shape (ld ldy).  The columns of H X
// and H^T X are independent, so with 128 columns or more the call runs in up
// to four column chunks: chunk c + 1 is copied in while chunk c is multiplied
// and chunk c - 1 copied out (two copy streams and the library stream, ordered
// by events; with pinned host buffers the PCIe transfers in both directions
// overlap the products).  Option host_chunks = 1 runs the call in one piece;
// a larger value sets the number of chunks.
void host_product(DeviceTree &t, ProdOp op, const double *X, long long xr, long long xc,
                  long long ldx, double *Y, long long ldy) {
  cudaStream_t s = lib_stream();
  DevBuf dx(xr * xc, s), dy(xr * xc, s);
  // option "matmat_precision" = 1 routes H X, H^T X and X H through the int8
  // tensor-core path (about 42 bits); the default keeps FP64 throughout
  bool aligned = true;
  for (int m : t.g.leaf_m) aligned = aligned && (m % 32 == 0);
  const bool mixed = aligned && option("matmat_precision", 0.0) == 1.0;
  auto product = [&](const double *xd, double *yd, int k) {
    if (mixed)
      product_mixed_op(t, op, xd, k, xr, yd, xr, s);
    else
      product_f64(t, op, xd, k, xr, yd, xr, s);
  };
  long long chunks = (op != ProdOp::L && xc >= 128) ? std::min<long long>(4, xc / 64) : 1;
  const double opt = option("host_chunks", 0.0);
  if (opt >= 1.0 && op != ProdOp::L) chunks = std::max(1LL, std::min((long long)opt, xc));
  if (chunks <= 1 || xr == 0) {
    h2d(dx.p, X, xr, xc, ldx, s);
    product(dx.p, dy.p, (int)(op == ProdOp::L ? xr : xc));
    d2h(Y, ldy, dy.p, xr, xc, s);
    HB_CUDA(cudaStreamSynchronize(s));
    return;
  }
  cudaStream_t si = copy_stream(0), so = copy_stream(1);
  Events ev(2 * chunks + 2);
  cudaEvent_t *in = ev.e.data(), *done = ev.e.data() + chunks;
  cudaEvent_t allocated = ev.e[2 * chunks], copied_out = ev.e[2 * chunks + 1];
  // the buffers are stream-ordered allocations of s
  HB_CUDA(cudaEventRecord(allocated, s));
  HB_CUDA(cudaStreamWaitEvent(si, allocated, 0));
  HB_CUDA(cudaStreamWaitEvent(so, allocated, 0));
  const long long per = (xc + chunks - 1) / chunks;
  try {
    for (long long c = 0; c < chunks; ++c) {
      const long long c0 = c * per, c1 = std::min(xc, c0 + per);
      if (c0 >= c1) break;
      h2d(dx.p + c0 * xr, X + c0 * ldx, xr, c1 - c0, ldx, si);
      HB_CUDA(cudaEventRecord(in[c], si));
      HB_CUDA(cudaStreamWaitEvent(s, in[c], 0));
      product(dx.p + c0 * xr, dy.p + c0 * xr, (int)(c1 - c0));
      HB_CUDA(cudaEventRecord(done[c], s));
      HB_CUDA(cudaStreamWaitEvent(so, done[c], 0));
      d2h(Y + c0 * ldy, ldy, dy.p + c0 * xr, xr, c1 - c0, so);
    }
  } catch (...) {
    // no copy may still use the buffers when they are freed
    cudaStreamSynchronize(si);
    cudaStreamSynchronize(so);
    throw;
  }
  // the buffers are freed on s after the last copy out
  HB_CUDA(cudaEventRecord(copied_out, so));
  HB_CUDA(cudaStreamWaitEvent(s, copied_out, 0));
  HB_CUDA(cudaStreamSynchronize(s));
}

std::shared_ptr<DeviceTree> subtree_device(const HODLRInternalNode *internal, int height,
                                           cudaStream_t s) {
  Geometry g = geometry_of_subtree(internal, height);
  std::shared_ptr<DeviceTree> dt = dtree_create(g, s);
  dtree_upload(*dt, const_cast<HODLRInternalNode *>(internal), s);
  return dt;
}

}  // namespace

extern "C" const char *hb_source_hash(void);

extern "C" {

// ------------------------------------------------------------ construction

int dense_to_tree_hodlr(TreeHODLR *hodlr, const int m, const int *ms, double *matrix,
                        const double svd_threshold, int *ierr) {
  if (hodlr == nullptr || matrix == nullptr) {
    *ierr = INPUT_ERROR;
    return 0;
  }
  *ierr = SUCCESS;
  try {
    const int h = hodlr->height;
    std::vector<int> leaf;
    if (ms == nullptr) {
      leaf = halves(m, h);
    } else {
      leaf.assign(ms, ms + (1 << h));
      long long total = 0;
      for (int v : leaf) {
        HB_REQUIRE(v >= 0, INPUT_ERROR, "negative block size");
        total += v;
      }
      apply_sizes(hodlr, leaf);
      if (total != m) {
        *ierr = INPUT_ERROR;   // hmat_lib src/constructors.c:652-655
        set_last_error("block sizes do not add up to m");
        return 0;
      }
    }
    apply_sizes(hodlr, leaf);
    Geometry g = geometry_of(hodlr);
    cudaStream_t s = lib_stream();
    DevBuf da((size_t)m * m, s);
    h2d(da.p, matrix, m, m, m, s);
    int status = SUCCESS;
    std::shared_ptr<DeviceTree> dt = build_from_dense(g, da.p, m, svd_threshold, s, &status);
    dtree_download(*dt, hodlr, s);
    register_device_tree(hodlr, dt);
    if (status != SUCCESS) {
      *ierr = status;
      // a sketch that reached its cap keeps the build's own message (which
      // cap, and the memory it saw)
      if (!last_build_stats().cap_hit)
        set_last_error("Jacobi SVD did not converge within the sweep limit");
      return 1;
    }
    return 0;
  } catch (const Error &e) {
    fail(ierr, e);
    return 0;
  }
}

// ---------------------------------------------------------------- products

double *multiply_vector(const TreeHODLR *hodlr, const double *vector, double *out, int *ierr) {
  if (hodlr == nullptr || vector == nullptr || vector == out) {
    *ierr = INPUT_ERROR;
    return nullptr;
  }
  bool owned = false;
  try {
    const int n = hodlr->root ? geometry_of(hodlr).n : 0;
    if (out == nullptr) {
      out = (double *)host_malloc((size_t)n * sizeof(double));
      if (out == nullptr) {
        *ierr = ALLOCATION_FAILURE;
        return nullptr;
      }
      owned = true;
    }
    *ierr = SUCCESS;
    auto dt = device_tree_for(hodlr, lib_stream());
    host_product(*dt, ProdOp::N, vector, n, 1, n, out, n);
    return out;
  } catch (const Error &e) {
    fail(ierr, e);
    if (owned) host_free(out);
    return nullptr;
  }
}

int compute_multiply_hodlr_dense_workspace(const TreeHODLR *hodlr, const int matrix_a) {
  return get_highest_s(hodlr) * matrix_a;
}

static double *dense_entry(const TreeHODLR *hodlr, ProdOp op, const double *matrix, int k,
                           int matrix_ld, double *out, int out_ld, int *ierr) {
  if (hodlr == nullptr || matrix == nullptr || matrix == out) {
    *ierr = INPUT_ERROR;
    return nullptr;
  }
  bool owned = false;
  try {
    const int n = geometry_of(hodlr).n;
    const long long cols = (op == ProdOp::L) ? n : k;   // columns of out
    if (out == nullptr) {
      out = (double *)host_malloc((size_t)std::max<long long>((long long)out_ld * cols, 1) *
                                  sizeof(double));
      if (out == nullptr) {
        *ierr = ALLOCATION_FAILURE;
        return nullptr;
      }
      owned = true;
    }
    *ierr = SUCCESS;
    auto dt = device_tree_for(hodlr, lib_stream());
    if (op == ProdOp::L)
      host_product(*dt, op, matrix, k, n, matrix_ld, out, out_ld);
    else
      host_product(*dt, op, matrix, n, k, matrix_ld, out, out_ld);
    return out;
  } catch (const Error &e) {
    fail(ierr, e);
    if (owned) host_free(out);
    return nullptr;
  }
}

double *multiply_hodlr_dense(const TreeHODLR *hodlr, const double *matrix, const int matrix_n,
                             const int matrix_ld, double *out, const int out_ld, int *ierr) {
  return dense_entry(hodlr, ProdOp::N, matrix, matrix_n, matrix_ld, out, out_ld, ierr);
}

double *multiply_hodlr_transpose_dense(const TreeHODLR *hodlr, const double *matrix,
                                       const int matrix_n, const int matrix_ld, double *out,
                                       const int out_ld, int *ierr) {
  return dense_entry(hodlr, ProdOp::T, matrix, matrix_n, matrix_ld, out, out_ld, ierr);
}

double *multiply_dense_hodlr(const TreeHODLR *hodlr, const double *matrix, const int matrix_m,
                             const int matrix_ld, double *out, const int out_ld, int *ierr) {
  return dense_entry(hodlr, ProdOp::L, matrix, matrix_m, matrix_ld, out, out_ld, ierr);
}

// Subtree products have no ierr in hmat_lib; failures are reported through
// hodlr_b200_last_error() and leave `out` unchanged.
static void internal_entry(const HODLRInternalNode *internal, int height, ProdOp op,
                           const double *matrix, int k, int matrix_ld, double *out, int out_ld) {
  if (internal == nullptr || matrix == nullptr || out == nullptr) {
    set_last_error("NULL argument");
    return;
  }
  try {
    cudaStream_t s = lib_stream();
    auto dt = subtree_device(internal, height, s);
    const int n = dt->g.n;
    if (op == ProdOp::L)
      host_product(*dt, op, matrix, k, n, matrix_ld, out, out_ld);
    else
      host_product(*dt, op, matrix, n, k, matrix_ld, out, out_ld);
  } catch (const Error &e) {
    set_last_error(e.msg);
  }
}

void multiply_internal_node_dense(const HODLRInternalNode *internal, const int height,
                                  const double *matrix, const int matrix_n, const int matrix_ld,
                                  const HODLRInternalNode **, double *, double *out,
                                  const int out_ld) {
  internal_entry(internal, height, ProdOp::N, matrix, matrix_n, matrix_ld, out, out_ld);
}

void multiply_internal_node_transpose_dense(const HODLRInternalNode *internal, const int height,
                                            const double *matrix, const int matrix_n,
                                            const int matrix_ld, const HODLRInternalNode **,
                                            double *, double *out, const int out_ld) {
  internal_entry(internal, height, ProdOp::T, matrix, matrix_n, matrix_ld, out, out_ld);
}

void multiply_dense_internal_node(const HODLRInternalNode *internal, const int height,
                                  const double *matrix, const int matrix_m, const int matrix_ld,
                                  const HODLRInternalNode **, double *, double *out,
                                  const int out_ld) {
  internal_entry(internal, height, ProdOp::L, matrix, matrix_m, matrix_ld, out, out_ld);
}

// ------------------------------------------------------------ HODLR x HODLR

int multiply_hodlr_hodlr(const TreeHODLR *hodlr1, const TreeHODLR *hodlr2, TreeHODLR *out,
                         const double svd_threshold, int *ierr) {
  if (hodlr1 == nullptr || hodlr2 == nullptr || out == nullptr) {
    *ierr = INPUT_ERROR;
    return 0;
  }
  *ierr = SUCCESS;
  try {
    HB_REQUIRE(hodlr1->height == hodlr2->height && out->height == hodlr1->height, INPUT_ERROR,
               "trees of different heights");
    cudaStream_t s = lib_stream();
    auto a = device_tree_for(hodlr1, s);
    auto b = device_tree_for(hodlr2, s);
    int status = SUCCESS;
    std::shared_ptr<DeviceTree> c = hxh_multiply(*a, *b, svd_threshold, s, &status);
    dtree_download(*c, out, s);
    register_device_tree(out, c);
    if (status != SUCCESS) {
      *ierr = status;
      set_last_error("SVD of a recompression did not converge");
      return 1;
    }
    return 0;
  } catch (const Error &e) {
    fail(ierr, e);
    return 0;
  }
}

// ------------------------------------------------------------ extensions

const char *hodlr_b200_version(void) {
  // hb_source_hash(): digest of the sources this binary was built from,
  // generated at build time (hmat_lib_b200/build.py)
  static const std::string v = std::string("hodlr-b200 0.2 (sm_100a) sources ") + hb_source_hash();
  return v.c_str();
}
const char *hodlr_b200_last_error(void) { return last_error(); }
long long hodlr_b200_kernel_launches(void) { return launches(); }

int hodlr_b200_set_option(const char *name, double value) {
  if (!name) return INPUT_ERROR;
  set_option(name, value);
  return SUCCESS;
}

void hodlr_b200_set_host_allocator(void *(*alloc_fn)(size_t), void (*free_fn)(void *)) {
  HostAllocator &a = host_allocator();
  if (alloc_fn && free_fn) {
    a.alloc = alloc_fn;
    a.release = free_fn;
  } else {
    a.alloc = &std::malloc;
    a.release = &std::free;
  }
}

int hodlr_b200_build_dev(int height, int n, const int *ms, const double *d_matrix, int ld,
                         double svd_threshold, int flags, void *stream, hodlr_b200_tree *out,
                         int *ierr) {
  (void)flags;
  if (!d_matrix || !out || height < 1 || n < 0) {
    if (ierr) *ierr = INPUT_ERROR;
    return INPUT_ERROR;
  }
  try {
    std::vector<int> leaf = ms ? std::vector<int>(ms, ms + (1 << height)) : halves(n, height);
    Geometry g = geometry_from_leaves(height, leaf);
    HB_REQUIRE(g.n == n, INPUT_ERROR, "block sizes do not add up to n");
    int status = SUCCESS;
    auto dt = build_from_dense(g, d_matrix, ld, svd_threshold, as_stream(stream), &status);
    *out = new hodlr_b200_tree_s{dt};
    if (ierr) *ierr = status;
    return status;
  } catch (const Error &e) {
    return fail(ierr, e);
  }
}

int hodlr_b200_build_batched_dev(int count, const int *heights, const int *ns,
                                 const double *const *d_matrices, const int *lds,
                                 double svd_threshold, void *stream, hodlr_b200_tree *out,
                                 int *ierr) {
  if (count < 0 || (count > 0 && (!heights || !ns || !d_matrices || !lds || !out))) {
    if (ierr) *ierr = INPUT_ERROR;
    return INPUT_ERROR;
  }
  if (count == 0) {
    if (ierr) *ierr = SUCCESS;
    return SUCCESS;
  }
  try {
    std::vector<BuildInput> in;
    for (int i = 0; i < count; ++i) {
      HB_REQUIRE(heights[i] >= 1 && ns[i] >= 0 && d_matrices[i] && lds[i] >= std::max(ns[i], 1),
                 INPUT_ERROR, "batched build: a tree with an invalid height, size or input");
      Geometry g = geometry_from_leaves(heights[i], halves(ns[i], heights[i]));
      in.push_back(BuildInput{g, d_matrices[i], lds[i]});
    }
    int status = SUCCESS;
    auto dts = build_batch(in, svd_threshold, as_stream(stream), &status);
    for (int i = 0; i < count; ++i) out[i] = new hodlr_b200_tree_s{dts[i]};
    if (ierr) *ierr = status;
    return status;
  } catch (const Error &e) {
    return fail(ierr, e);
  }
}

void hodlr_b200_tree_free(hodlr_b200_tree t) { delete t; }

int hodlr_b200_tree_to_host(hodlr_b200_tree t, TreeHODLR *hodlr, int *ierr) {
  if (!t || !hodlr || hodlr->height != t->p->g.h) {
    if (ierr) *ierr = INPUT_ERROR;
    return INPUT_ERROR;
  }
  try {
    dtree_download(*t->p, hodlr, lib_stream());
    register_device_tree(hodlr, t->p);
    if (ierr) *ierr = SUCCESS;
    return SUCCESS;
  } catch (const Error &e) {
    return fail(ierr, e);
  }
}

int hodlr_b200_build_kernel_dev(int height, int n, const int *ms, const double *d_points,
                                int dim, int kind, double length, double diag,
                                double svd_threshold, int flags, void *stream,
                                hodlr_b200_tree *out, int *ierr) {
  (void)flags;
  if (!d_points || !out || height < 1 || n < 0 || dim < 1 || kind < 0 || kind > 2 ||
      !(length > 0.0)) {
    if (ierr) *ierr = INPUT_ERROR;
    return INPUT_ERROR;
  }
  try {
    std::vector<int> leaf = ms ? std::vector<int>(ms, ms + (1 << height)) : halves(n, height);
    Geometry g = geometry_from_leaves(height, leaf);
    HB_REQUIRE(g.n == n, INPUT_ERROR, "block sizes do not add up to n");
    KernelSpec K;
    K.pts = d_points;
    K.n = n;
    K.dim = dim;
    K.kind = kind;
    K.length = length;
    K.diag = diag;
    int status = SUCCESS;
    auto dt = build_from_dense(g, nullptr, n, svd_threshold, as_stream(stream), &status,
                               nullptr, &K);
    *out = new hodlr_b200_tree_s{dt};
    if (ierr) *ierr = status;
    return status;
  } catch (const Error &e) {
    return fail(ierr, e);
  }
}

}  // extern "C"

struct hodlr_b200_factor_s {
  std::unique_ptr<HodlrFactor> f;
};

extern "C" {

int hodlr_b200_factorize_dev(hodlr_b200_tree t, void *stream, hodlr_b200_factor *out, int *ierr) {
  if (!t || !out) {
    if (ierr) *ierr = INPUT_ERROR;
    return INPUT_ERROR;
  }
  try {
    int status = SUCCESS;
    auto f = hodlr_factorize(t->p, as_stream(stream), &status);
    if (status != SUCCESS) {
      set_last_error("factorisation: a leaf or capacitance matrix is singular to working precision");
      if (ierr) *ierr = status;
      return status;
    }
    *out = new hodlr_b200_factor_s{std::move(f)};
    if (ierr) *ierr = SUCCESS;
    return SUCCESS;
  } catch (const Error &e) {
    return fail(ierr, e);
  }
}

int hodlr_b200_solve_dev(hodlr_b200_factor f, const double *d_b, int k, int ldb, double *d_x,
                         int ldx, void *stream) {
  if (!f || !d_b || !d_x || d_b == d_x || k < 0) return INPUT_ERROR;
  try {
    const int n = f->f->tree->g.n;
    HB_REQUIRE(ldb >= std::max(1, n) && ldx >= std::max(1, n), INPUT_ERROR,
               "leading dimension below n");
    hodlr_solve(*f->f, d_b, k, ldb, d_x, ldx, as_stream(stream));
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

void hodlr_b200_factor_free(hodlr_b200_factor f) { delete f; }

hodlr_b200_tree hodlr_b200_tree_from_host(const TreeHODLR *hodlr, int *ierr) {
  try {
    auto dt = device_tree_for(hodlr, lib_stream());
    if (ierr) *ierr = SUCCESS;
    return new hodlr_b200_tree_s{dt};
  } catch (const Error &e) {
    fail(ierr, e);
    return nullptr;
  }
}

int hodlr_b200_tree_info(hodlr_b200_tree t, int *height, int *n, int *max_rank,
                         long long *storage_doubles, long long *arena_bytes) {
  if (!t) return INPUT_ERROR;
  if (height) *height = t->p->g.h;
  if (n) *n = t->p->g.n;
  if (max_rank) *max_rank = t->p->g.max_rank();
  if (storage_doubles) *storage_doubles = t->p->storage();
  if (arena_bytes) *arena_bytes = t->p->arena_elems * (long long)sizeof(double);
  return SUCCESS;
}

int hodlr_b200_tree_ranks(hodlr_b200_tree t, int *ranks, int capacity) {
  if (!t) return -1;
  const int nb = t->p->g.nblock();
  for (int b = 0; b < nb && b < capacity; ++b) ranks[b] = t->p->g.blocks[b].s;
  return nb;
}

int hodlr_b200_matmat_dev(hodlr_b200_tree t, int op, int precision, const double *d_x, int k,
                          int ldx, double *d_y, int ldy, void *stream) {
  if (!t || !d_x || !d_y || op < 0 || op > 2) return INPUT_ERROR;
  try {
    const long long rows = (op == HODLR_B200_OP_L) ? k : t->p->g.n;
    HB_REQUIRE(k >= 0 && ldx >= std::max(1LL, rows) && ldy >= std::max(1LL, rows), INPUT_ERROR,
               "leading dimension below the number of rows");
    if (precision == HODLR_B200_MIXED) {
      product_mixed_op(*t->p, (ProdOp)op, d_x, k, ldx, d_y, ldy, as_stream(stream));
      return SUCCESS;
    }
    HB_REQUIRE(precision == HODLR_B200_FP64, INPUT_ERROR, "unknown precision mode");
    product_f64(*t->p, (ProdOp)op, d_x, k, ldx, d_y, ldy, as_stream(stream));
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_hxh_dev(hodlr_b200_tree a, hodlr_b200_tree b, double svd_threshold,
                       hodlr_b200_tree *out, int *ierr) {
  if (!a || !b || !out) {
    if (ierr) *ierr = INPUT_ERROR;
    return INPUT_ERROR;
  }
  try {
    int status = SUCCESS;
    auto c = hxh_multiply(*a->p, *b->p, svd_threshold, lib_stream(), &status);
    *out = new hodlr_b200_tree_s{c};
    if (ierr) *ierr = status;
    return status;
  } catch (const Error &e) {
    return fail(ierr, e);
  }
}

int hodlr_b200_recompress_dev(int m, int n, int s, const double *d_u, int ldu, const double *d_v,
                              int ldv, double svd_threshold, int dense, double *d_u_out,
                              double *d_v_out, int *rank, void *stream) {
  if (!rank) return INPUT_ERROR;
  try {
    return recompress_one(m, n, s, d_u, ldu, d_v, ldv, svd_threshold, dense != 0, d_u_out,
                          d_v_out, rank, as_stream(stream));
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_phase_times(double *out, int capacity) { return phase_times(out, capacity); }

int hodlr_b200_check(hodlr_b200_tree t, void *stream) {
  if (!t) return INPUT_ERROR;
  try {
    if (mixed_status(*t->p, as_stream(stream)) != 0) {
      set_last_error("a mixed-precision kernel gave up waiting on a barrier");
      return SVD_FAILURE;
    }
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_matmat_batched_dev(int count, const hodlr_b200_tree *trees, int op, int precision,
                                  const double *const *d_x, const int *k, const int *ldx,
                                  double *const *d_y, const int *ldy, void *stream) {
  if (count < 0 || (count > 0 && (!trees || !d_x || !k || !ldx || !d_y || !ldy)) || op < 0 ||
      op > 2)
    return INPUT_ERROR;
  try {
    HB_REQUIRE(precision == HODLR_B200_FP64 || precision == HODLR_B200_MIXED, INPUT_ERROR,
               "unknown precision mode");
    std::vector<std::shared_ptr<DeviceTree>> ts;
    std::vector<const double *> xs;
    std::vector<double *> ys;
    std::vector<int> ks;
    std::vector<long long> lx, ly;
    for (int i = 0; i < count; ++i) {
      HB_REQUIRE(trees[i] != nullptr, INPUT_ERROR, "batched product: NULL tree");
      ts.push_back(trees[i]->p);
      xs.push_back(d_x[i]);
      ys.push_back(d_y[i]);
      ks.push_back(k[i]);
      lx.push_back(ldx[i]);
      ly.push_back(ldy[i]);
    }
    batched_product(ts, (ProdOp)op, (Precision)precision, xs, ks, lx, ys, ly, as_stream(stream));
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_batched_tuning(char *buf, int capacity) {
  const std::string t = batched_tuning();
  if (buf && capacity > 0) {
    const size_t n = std::min<size_t>(t.size(), (size_t)capacity - 1);
    std::memcpy(buf, t.data(), n);
    buf[n] = 0;
  }
  return (int)t.size();
}

int hodlr_b200_batched_check(void) {
  try {
    if (batched_status() != 0) {
      set_last_error("a mixed-precision kernel gave up waiting on a barrier");
      return SVD_FAILURE;
    }
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

void hodlr_b200_batched_release(void) { batched_release(); }

// ---------------------------------------------------------------- rank model

namespace {
struct DevFloats {
  float *p = nullptr;
  cudaStream_t s;
  DevFloats(const float *host, size_t n, cudaStream_t st) : s(st) {
    HB_CUDA(cudaMallocAsync((void **)&p, sizeof(float) * std::max<size_t>(n, 1), s));
    if (host && n)
      HB_CUDA(cudaMemcpyAsync(p, host, sizeof(float) * n, cudaMemcpyHostToDevice, s));
  }
  void to_host(float *host, size_t n) {
    if (host && n) HB_CUDA(cudaMemcpyAsync(host, p, sizeof(float) * n, cudaMemcpyDeviceToHost, s));
  }
  ~DevFloats() { cudaFreeAsync(p, s); }
};
}  // namespace

int hodlr_b200_rank_model_size(void) { return kRankParams; }

int hodlr_b200_rank_model_set(const float *params, int count) {
  if (count == 0) {
    set_rank_model({});
    return SUCCESS;
  }
  if (!params || count != kRankParams) {
    set_last_error("rank model: wrong parameter count");
    return INPUT_ERROR;
  }
  set_rank_model(std::vector<float>(params, params + count));
  return SUCCESS;
}

int hodlr_b200_rank_model_get(float *params, int capacity) {
  std::vector<float> m;
  if (!rank_model(m)) return 0;
  if (params) std::copy(m.begin(), m.begin() + std::min<int>(capacity, (int)m.size()), params);
  return (int)m.size();
}

int hodlr_b200_rank_model_train(const float *features, const float *targets, int n, int steps,
                                int batch, double lr, unsigned long long seed, float *params_out,
                                float *loss_log, int log_capacity) {
  if (!features || !targets || !params_out || n <= 0 || steps <= 0 || batch <= 0)
    return INPUT_ERROR;
  try {
    RankTrainConfig cfg;
    cfg.steps = steps;
    cfg.batch = batch;
    cfg.lr = (float)lr;
    cfg.seed = seed;
    std::vector<float> loss;
    std::vector<float> P = rank_mlp_train(std::vector<float>(features, features + (size_t)n * kRankIn),
                                          std::vector<float>(targets, targets + n), cfg, &loss,
                                          lib_stream());
    std::copy(P.begin(), P.end(), params_out);
    for (int i = 0; loss_log && i < log_capacity && i < (int)loss.size(); ++i) loss_log[i] = loss[i];
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_rank_model_predict(const float *params, const float *features, int n, float *out) {
  if (!params || !features || !out || n < 0) return INPUT_ERROR;
  try {
    cudaStream_t s = lib_stream();
    DevFloats dp(params, kRankParams, s), dx(features, (size_t)n * kRankIn, s), dy(nullptr, n, s);
    rank_mlp_predict(dp.p, dx.p, n, dy.p, s);
    dy.to_host(out, n);
    HB_CUDA(cudaStreamSynchronize(s));
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_rank_model_gradient(const float *params, const float *features,
                                   const float *targets, int n, float *grad_out,
                                   float *loss_out) {
  if (!params || !features || !targets || !grad_out || n <= 0) return INPUT_ERROR;
  try {
    cudaStream_t s = lib_stream();
    DevFloats dp(params, kRankParams, s), dx(features, (size_t)n * kRankIn, s),
        dt(targets, n, s), dg(nullptr, kRankParams, s), dl(nullptr, 1, s);
    rank_mlp_gradient(dp.p, dx.p, dt.p, n, dg.p, dl.p, s);
    dg.to_host(grad_out, kRankParams);
    dl.to_host(loss_out, loss_out ? 1 : 0);
    HB_CUDA(cudaStreamSynchronize(s));
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_rank_model_adam(float *params, const float *grad, float *m, float *v, int step,
                               double lr) {
  if (!params || !grad || !m || !v || step < 1) return INPUT_ERROR;
  try {
    cudaStream_t s = lib_stream();
    DevFloats dp(params, kRankParams, s), dg(grad, kRankParams, s), dm(m, kRankParams, s),
        dv(v, kRankParams, s);
    RankTrainConfig cfg;
    cfg.lr = (float)lr;
    rank_mlp_adam(dp.p, dg.p, dm.p, dv.p, step, cfg, s);
    dp.to_host(params, kRankParams);
    dm.to_host(m, kRankParams);
    dv.to_host(v, kRankParams);
    HB_CUDA(cudaStreamSynchronize(s));
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

int hodlr_b200_build_features(float *out, int capacity_rows) {
  const std::vector<float> &f = last_build_features();
  const int rows = (int)(f.size() / kFeatureRow);
  if (out)
    std::copy(f.begin(), f.begin() + (size_t)std::min(rows, std::max(capacity_rows, 0)) * kFeatureRow,
              out);
  return rows;
}

int hodlr_b200_build_stats(double *out, int capacity) {
  const BuildStats &st = last_build_stats();
  const double v[] = {(double)st.exact_blocks,     (double)st.sketched_blocks,
                      (double)st.sketch_rounds,    st.seconds,
                      (double)st.cap_hit,          (double)st.max_sweeps_exact,
                      (double)st.max_sweeps_sketch, (double)st.failed_exact,
                      (double)st.failed_sketch,    (double)st.max_sketch,
                      st.ms_exact,                 st.ms_rounds,
                      st.ms_core_svd,              st.ms_finish,
                      (double)st.learned_fallbacks, st.ms_features,
                      st.gemm_flops,               st.input_elems,
                      st.ms_host_setup,            st.ms_host_plans};
  const int n = (int)(sizeof(v) / sizeof(v[0]));
  for (int i = 0; i < n && i < capacity && out; ++i) out[i] = v[i];
  return n;
}

int hodlr_b200_sync_tree(const TreeHODLR *hodlr) {
  try {
    forget_device_tree(hodlr);
    device_tree_for(hodlr, lib_stream());
    return SUCCESS;
  } catch (const Error &e) {
    return fail(nullptr, e);
  }
}

}  // extern "C"
