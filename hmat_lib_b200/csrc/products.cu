// HODLR x dense products (FP64) built on the segmented GEMM engine.
//
// Replaces hmat_lib src/dense_algebra.c (multiply_hodlr_dense :361,
// multiply_hodlr_transpose_dense :617, multiply_dense_hodlr :957 and the
// subtree variants :492, :710, :1087) and src/vector_algebra.c:131
// (multiply_vector, the k = 1 case).  The reference walks the tree block by
// block with two dgemm calls per block; here all blocks of all levels run in
// two launches.
#include "products.h"

namespace hb {

namespace {
enum Base { kArena = 0, kX = 1, kY = 2, kW = 3 };
}

ProductPlan::~ProductPlan() {
  if (w) cudaFree(w);
}

ProductWork product_work(const DeviceTree &t, int k) {
  ProductWork w{};
  w.elements = (double)t.storage();
  w.flops = 2.0 * k * w.elements;
  w.bytes = 8.0 * w.elements + 16.0 * (double)t.g.n * k;
  return w;
}

// block (of the node containing leaf i at depth d) whose rows (row_side) or
// columns (!row_side) cover leaf i
static int covering_block(int h, int i, int d, bool row_side) {
  const int j = i >> (h - d);
  const bool top = ((i >> (h - d - 1)) & 1) == 0;
  int c;
  if (row_side)
    c = top ? 1 : 2;
  else
    c = top ? 2 : 1;
  return block_index(d, j, c);
}

void append_product(GemmBatch &p1, GemmBatch &p2, const DeviceTree &t, ProdOp op, int k,
                    long long ldx, long long ldy, const ProductSlots &sl,
                    const std::vector<long long> &w_off, int min_depth) {
  const Geometry &g = t.g;
  const int h = g.h;
  const int A = sl.arena, X = sl.x, Y = sl.y, W = sl.w;
  const long long ao = sl.arena_off, xo = sl.x_off, yo = sl.y_off, wo = sl.w_off;
  // phase 1: projections
  for (size_t bi = 0; bi < g.blocks.size(); ++bi) {
    const BlockDesc &b = g.blocks[bi];
    if (b.s == 0 || b.depth < min_depth) continue;
    if (op == ProdOp::N) {          // W_b (s x k) = V_b^T X[c0 : c0 + n]
      int p = p1.add(W, wo + w_off[bi], b.s, b.s, k);
      p1.seg(p, A, ao + b.v_off, b.n, 1, X, xo + b.c0, ldx, 0, b.n);
    } else if (op == ProdOp::T) {   // W_b (s x k) = U_b^T X[r0 : r0 + m]
      int p = p1.add(W, wo + w_off[bi], b.s, b.s, k);
      p1.seg(p, A, ao + b.u_off, b.m, 1, X, xo + b.r0, ldx, 0, b.m);
    } else {                        // Z_b (k x s) = X[:, r0 : r0 + m] U_b
      int p = p1.add(W, wo + w_off[bi], k, k, b.s);
      p1.seg(p, X, xo + (long long)b.r0 * ldx, ldx, 0, A, ao + b.u_off, b.m, 0, b.m);
    }
  }
  // phase 2: one problem per leaf row band (columns for op L)
  for (int i = 0; i < g.nleaf(); ++i) {
    const LeafDesc &L = t.leaves[i];
    if (L.m == 0) continue;
    if (op == ProdOp::N || op == ProdOp::T) {
      int p = p2.add(Y, yo + L.r0, ldy, L.m, k);
      p2.seg(p, A, ao + L.off, L.m, op == ProdOp::T ? 1 : 0, X, xo + L.r0, ldx, 0, L.m);
      for (int d = h - 1; d >= min_depth; --d) {
        const int bi = covering_block(h, i, d, op == ProdOp::N);
        const BlockDesc &b = g.blocks[bi];
        if (b.s == 0) continue;
        if (op == ProdOp::N)
          p2.seg(p, A, ao + b.u_off + (L.r0 - b.r0), b.m, 0, W, wo + w_off[bi], b.s, 0, b.s);
        else
          p2.seg(p, A, ao + b.v_off + (L.r0 - b.c0), b.n, 0, W, wo + w_off[bi], b.s, 0, b.s);
      }
    } else {
      int p = p2.add(Y, yo + (long long)L.r0 * ldy, ldy, k, L.m);
      p2.seg(p, X, xo + (long long)L.r0 * ldx, ldx, 0, A, ao + L.off, L.m, 0, L.m);
      for (int d = h - 1; d >= min_depth; --d) {
        const int bi = covering_block(h, i, d, false);
        const BlockDesc &b = g.blocks[bi];
        if (b.s == 0) continue;
        p2.seg(p, W, wo + w_off[bi], k, 0, A, ao + b.v_off + (L.r0 - b.c0), b.n, 1, b.s);
      }
    }
  }
}

long long product_w_layout(const DeviceTree &t, int k, std::vector<long long> &w_off) {
  long long w_total = 0;
  w_off.assign(t.g.blocks.size(), 0);
  for (size_t b = 0; b < t.g.blocks.size(); ++b) {
    w_off[b] = w_total;
    w_total += align_up((long long)t.g.blocks[b].s * k);
  }
  return w_total;
}

// Tile shape of a product phase: option product_shape1 / product_shape2
// (0-3: 128x64, 64x128, 32x128, 32x256), else by op and k.
TileShape default_shape(ProdOp op, int k, int phase) {
  const int forced =
      (int)(phase == 1 ? option("product_shape1", -1.0) : option("product_shape2", -1.0));
  if (forced >= 0 && forced <= 3) return (TileShape)forced;
  if (phase == 1) return (op == ProdOp::L) ? TileShape::M128N64 : TileShape::M64N128;
  return (op == ProdOp::L && k <= 64) ? TileShape::M64N128 : TileShape::M128N64;
}

ProductPlan &product_plan(DeviceTree &t, ProdOp op, int k, long long ldx, long long ldy,
                          cudaStream_t stream, int min_depth) {
  std::lock_guard<std::mutex> lk(t.plan_mutex);
  // the tile shapes are part of the key (precision field: FP64 plus the shapes)
  const int shapes = 16 * (1 + (int)default_shape(op, k, 1)) + 256 * (1 + (int)default_shape(op, k, 2));
  auto key = std::make_tuple((int)op, k, ldx, ldy, (int)Precision::FP64 + shapes, min_depth);
  auto it = t.plans.find(key);
  if (it != t.plans.end()) return *it->second;

  auto plan = std::make_unique<ProductPlan>();
  plan->op = op;
  plan->k = k;
  plan->ldx = ldx;
  plan->ldy = ldy;
  std::vector<long long> w_off;
  const long long w_total = product_w_layout(t, k, w_off);
  plan->w_elems = w_total;
  HB_CUDA(cudaMalloc(&plan->w, std::max<long long>(w_total, 1) * sizeof(double)));
  GemmBatch p1, p2;
  append_product(p1, p2, t, op, k, ldx, ldy, ProductSlots{kArena, kX, kY, kW, 0, 0, 0, 0}, w_off,
                 min_depth);
  if (!p1.empty()) gemm_plan_build(plan->phase1, p1, default_shape(op, k, 1), true, stream);
  if (!p2.empty()) gemm_plan_build(plan->phase2, p2, default_shape(op, k, 2), false, stream);
  auto &ref = *plan;
  t.plans[key] = std::move(plan);
  return ref;
}

// Optional per-phase timing: with option "record_phase_times" set, events are
// recorded on the launching stream around each phase and their elapsed times
// accumulated (read and reset with hodlr_b200_phase_times).  Work is never
// skipped; the events only bracket it.
namespace {
std::mutex g_pt_mutex;
struct PhaseEvents {
  cudaEvent_t e[3];
  cudaEvent_t k[4];   // around the GEMM launch of each phase, when marked
  bool kmarks;
};
std::vector<PhaseEvents> g_pending;
double g_phase_ms[2] = {0.0, 0.0};
double g_kernel_ms[2] = {0.0, 0.0};
long long g_phase_count = 0;

void collect_phase_times() {
  for (auto &pe : g_pending) {
    cudaEventSynchronize(pe.e[2]);
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, pe.e[0], pe.e[1]);
    cudaEventElapsedTime(&b, pe.e[1], pe.e[2]);
    g_phase_ms[0] += a;
    g_phase_ms[1] += b;
    if (pe.kmarks) {
      float c = 0.f, d = 0.f;
      cudaEventElapsedTime(&c, pe.k[0], pe.k[1]);
      cudaEventElapsedTime(&d, pe.k[2], pe.k[3]);
      g_kernel_ms[0] += c;
      g_kernel_ms[1] += d;
    } else {            // the phase is its GEMM launch
      g_kernel_ms[0] += a;
      g_kernel_ms[1] += b;
    }
    g_phase_count += 1;
    for (auto ev : pe.e) cudaEventDestroy(ev);
    for (auto ev : pe.k) cudaEventDestroy(ev);
  }
  g_pending.clear();
}
}  // namespace

PhaseTimer::PhaseTimer(cudaStream_t s) : stream(s) {
  on = option("record_phase_times", 0.0) != 0.0;
  if (!on) return;
  for (auto &ev : e) HB_CUDA(cudaEventCreate(&ev));
  for (auto &ev : k) HB_CUDA(cudaEventCreate(&ev));
  HB_CUDA(cudaEventRecord(e[0], stream));
}

void PhaseTimer::kernel(int phase, bool end) {
  if (!on) return;
  kmarks = true;
  HB_CUDA(cudaEventRecord(k[2 * (phase - 1) + (end ? 1 : 0)], stream));
}

void PhaseTimer::mark(int i) {
  if (!on) return;
  HB_CUDA(cudaEventRecord(e[i], stream));
  if (i == 2) {
    std::lock_guard<std::mutex> lk(g_pt_mutex);
    g_pending.push_back(PhaseEvents{{e[0], e[1], e[2]}, {k[0], k[1], k[2], k[3]}, kmarks});
  }
}

int phase_times(double *out, int cap) {
  std::lock_guard<std::mutex> lk(g_pt_mutex);
  collect_phase_times();
  if (cap >= 1 && out) out[0] = g_phase_ms[0];
  if (cap >= 2 && out) out[1] = g_phase_ms[1];
  if (cap >= 3 && out) out[2] = (double)g_phase_count;
  if (cap >= 4 && out) out[3] = g_kernel_ms[0];
  if (cap >= 5 && out) out[4] = g_kernel_ms[1];
  g_phase_ms[0] = g_phase_ms[1] = 0.0;
  g_kernel_ms[0] = g_kernel_ms[1] = 0.0;
  g_phase_count = 0;
  return 5;
}

namespace {

// Runs `launch` (the kernel launches of one product) directly, or as a CUDA
// graph: the first call of a signature runs directly (lazy plans and scratch
// are made then), the second is captured on `stream` and replayed, later ones
// only replay.  Not with the legacy default stream, inside a caller's stream
// capture, with phase timing on, or with option product_graphs = 0.
template <class F>
void run_graphed(DeviceTree &t, ProdOp op, int k, long long ldx, long long ldy, int min_depth,
                 const double *X, double *Y, cudaStream_t stream, F launch) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool graphable = stream != nullptr && option("product_graphs", 1.0) != 0.0 &&
                         option("record_phase_times", 0.0) == 0.0 &&
                         cudaStreamIsCapturing(stream, &cs) == cudaSuccess &&
                         cs == cudaStreamCaptureStatusNone;
  if (!graphable) {
    (void)cudaGetLastError();
    launch();
    return;
  }
  const auto key = std::make_tuple((int)op, k, ldx, ldy, min_depth, (const void *)X, (void *)Y,
                                   (void *)stream);
  std::unique_ptr<ProductGraph> *slot;
  {
    std::lock_guard<std::mutex> lk(t.plan_mutex);
    auto it = t.graphs.find(key);
    if (it == t.graphs.end()) {
      if (t.graphs.size() >= 256) t.graphs.clear();   // bounded cache
      t.graphs.emplace(key, nullptr);                 // seen once
      slot = nullptr;
    } else {
      slot = &it->second;
    }
  }
  if (!slot) {
    launch();
    return;
  }
  if (!*slot) {
    const long long l0 = launches();
    cudaGraph_t graph = nullptr;
    HB_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      launch();
    } catch (...) {
      cudaStreamEndCapture(stream, &graph);
      if (graph) cudaGraphDestroy(graph);
      (void)cudaGetLastError();
      throw;
    }
    HB_CUDA(cudaStreamEndCapture(stream, &graph));
    auto pg = std::make_unique<ProductGraph>();
    pg->launches = launches() - l0;
    const cudaError_t e = cudaGraphInstantiate(&pg->exec, graph, 0);
    cudaGraphDestroy(graph);
    HB_CUDA(e);
    *slot = std::move(pg);
    // the captured launches were counted when captured; the replay below
    // counts them again as run
    count_launch(-(*slot)->launches);
  }
  HB_CUDA(cudaGraphLaunch((*slot)->exec, stream));
  count_launch((*slot)->launches);
}

}  // namespace

void product_f64(DeviceTree &t, ProdOp op, const double *X, int k, long long ldx, double *Y,
                 long long ldy, cudaStream_t stream, int min_depth) {
  if (k <= 0 || t.g.n == 0) return;
  run_graphed(t, op, k, ldx, ldy, min_depth, X, Y, stream,
              [&] { product_f64_direct(t, op, X, k, ldx, Y, ldy, stream, min_depth); });
}

void product_f64_direct(DeviceTree &t, ProdOp op, const double *X, int k, long long ldx, double *Y,
                        long long ldy, cudaStream_t stream, int min_depth) {
  if (k <= 0 || t.g.n == 0) return;
  // one vector: the HBM-bound matvec kernels (option matvec_kernels = 0 keeps
  // the GEMM engine)
  if (k == 1 && op == ProdOp::N && min_depth == 0 && option("matvec_kernels", 1.0) != 0.0) {
    PhaseTimer timer(stream);
    matvec_f64(t, X, Y, stream);
    timer.mark(1);
    timer.mark(2);
    return;
  }
  ProductPlan &plan = product_plan(t, op, k, ldx, ldy, stream, min_depth);
  GemmBases bases{};
  bases.p[kArena] = t.arena;
  bases.p[kX] = const_cast<double *>(X);
  bases.p[kY] = Y;
  bases.p[kW] = plan.w;
  bases.p[4] = t.arena;
  bases.p[5] = t.arena;
  PhaseTimer timer(stream);
  gemm_plan_run(plan.phase1, bases, stream);
  timer.mark(1);
  gemm_plan_run(plan.phase2, bases, stream);
  timer.mark(2);
}

}  // namespace hb
