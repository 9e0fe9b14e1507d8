// Products of many HODLR trees of uneven size and rank in one launch per
// phase (hodlr_b200_matmat_batched_dev).
//
// The reference multiplies one tree at a time, two dgemm calls per block
// (hmat_lib src/dense_algebra.c:361 multiply_hodlr_dense).  Here every block
// of every level of every tree is one problem of the same segmented GEMM
// launch: all operands are addressed as element offsets from one common base
// pointer (the lowest address among the trees' arenas, the inputs, the
// outputs and the batch's scratch), so the descriptors of all trees merge
// into one plan per phase.  Mixed precision merges the trees' int8 tile lists
// the same way (products_mixed.cu).
//
// A plan is made once per call signature (trees, pointers, sizes, op,
// precision) and kept in a small cache.  When it is made, the autotuner times
// every candidate configuration of each phase on the real operands (tile
// shape 128 x 64 or 64 x 128, with or without splitting long K ranges across
// tiles) and keeps the fastest; the chosen launches are then captured once
// into a CUDA graph that later calls replay.
#include <list>
#include <string>

#include "products.h"

namespace hb {

namespace {

struct BatchEntry {
  std::weak_ptr<DeviceTree> t;
  const DeviceTree *raw;
  const double *X;
  int k;
  long long ldx;
  double *Y;
  long long ldy;
};

struct BatchPlan {
  int op = 0, precision = 0, device = 0;
  std::vector<BatchEntry> sig;   // weak: a freed tree invalidates the plan, never kept alive
  // FP64
  std::unique_ptr<GemmPlan> ph1, ph2;
  double *w = nullptr;
  double *base = nullptr;
  // mixed
  std::unique_ptr<MixedBatch, MixedBatchDeleter> mixed;
  // replay
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long graph_launches = 0;
  std::string tuned;

  ~BatchPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    ph1.reset();
    ph2.reset();
    mixed.reset();
    if (w) cudaFree(w);
  }

  void run(cudaStream_t s) const {
    if (precision == (int)Precision::MIXED) {
      mixed_batch_run(*mixed, s);
      return;
    }
    GemmBases b{};
    for (int i = 0; i < kGemmBases; ++i) b.p[i] = base;
    if (ph1) gemm_plan_run(*ph1, b, s);
    if (ph2) gemm_plan_run(*ph2, b, s);
  }
};

std::mutex g_batch_mutex;
std::list<std::unique_ptr<BatchPlan>> g_batch_cache;   // most recent first
std::string g_last_tuned;
constexpr size_t kBatchCacheSize = 4;

bool same_signature(const BatchPlan &p, int op, int precision, int device,
                    const std::vector<BatchEntry> &sig) {
  if (p.op != op || p.precision != precision || p.device != device || p.sig.size() != sig.size())
    return false;
  for (size_t i = 0; i < sig.size(); ++i) {
    const BatchEntry &a = p.sig[i], &b = sig[i];
    if (a.t.expired() || a.raw != b.raw || a.X != b.X || a.k != b.k || a.ldx != b.ldx ||
        a.Y != b.Y || a.ldy != b.ldy)
      return false;
  }
  return true;
}

// Device time of `fn` on `s`: best of `reps` runs after one warm-up run.
template <class F>
float time_best(F fn, cudaStream_t s, int reps = 3) {
  cudaEvent_t a, b;
  HB_CUDA(cudaEventCreate(&a));
  HB_CUDA(cudaEventCreate(&b));
  fn();
  float best = 1e30f;
  for (int r = 0; r < reps; ++r) {
    HB_CUDA(cudaEventRecord(a, s));
    fn();
    HB_CUDA(cudaEventRecord(b, s));
    HB_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    HB_CUDA(cudaEventElapsedTime(&ms, a, b));
    best = std::min(best, ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

std::string shape_name(TileShape t) {
  return std::to_string(tile_rows(t)) + "x" + std::to_string(tile_cols(t));
}

// Plans phase `phase` of the FP64 batch for every candidate configuration,
// times them on the real operands, keeps the fastest.
std::unique_ptr<GemmPlan> tune_phase(const GemmBatch &batch, int phase, ProdOp op, int kmax,
                                     BatchPlan &P, cudaStream_t s, bool autotune) {
  if (batch.empty()) return nullptr;
  struct Cand {
    TileShape shape;
    bool split;
  };
  std::vector<Cand> cands;
  const int forced = (int)option("batch_shape", -1.0);   // 0..3: one shape, no timing
  if (forced >= 0 && forced <= 3) {
    cands.push_back(Cand{(TileShape)forced, phase == 1});
  } else if (autotune) {
    for (TileShape sh : {TileShape::M128N64, TileShape::M64N128, TileShape::M32N128,
                         TileShape::M32N256})
      for (bool sp : {false, true}) cands.push_back(Cand{sh, sp});
  } else {
    cands.push_back(Cand{default_shape(op, kmax, phase), phase == 1});
  }
  std::unique_ptr<GemmPlan> best;
  float best_ms = 1e30f;
  std::string best_desc;
  GemmBases b{};
  for (int i = 0; i < kGemmBases; ++i) b.p[i] = P.base;
  for (const Cand &c : cands) {
    GemmBatch copy = batch;
    auto plan = std::make_unique<GemmPlan>();
    gemm_plan_build(*plan, copy, c.shape, c.split, s);
    if (plan->ntiles == 0) continue;
    float ms = 0.f;
    if (cands.size() > 1) ms = time_best([&] { gemm_plan_run(*plan, b, s); }, s);
    if (!best || ms < best_ms) {
      best_ms = ms;
      best = std::move(plan);
      best_desc = std::string("phase") + std::to_string(phase) + " " + shape_name(c.shape) +
                  (best->any_split ? " split" : " nosplit") +
                  (cands.size() > 1 ? " " + std::to_string(ms) + " ms" : "");
    }
  }
  if (!P.tuned.empty()) P.tuned += "; ";
  P.tuned += best_desc;
  return best;
}

void build_fp64(BatchPlan &P, const std::vector<std::shared_ptr<DeviceTree>> &trees, ProdOp op,
                const std::vector<BatchEntry> &sig, cudaStream_t s, bool autotune) {
  const size_t n = trees.size();
  std::vector<std::vector<long long>> w_off(n);
  std::vector<long long> w_base(n, 0);
  long long w_total = 0;
  for (size_t i = 0; i < n; ++i) {
    w_base[i] = w_total;
    w_total += product_w_layout(*trees[i], sig[i].k, w_off[i]);
  }
  HB_CUDA(cudaMalloc(&P.w, std::max<long long>(w_total, 1) * sizeof(double)));
  const double *base = P.w;
  for (size_t i = 0; i < n; ++i)
    for (const double *p : {(const double *)trees[i]->arena, sig[i].X, (const double *)sig[i].Y})
      if (p < base) base = p;
  P.base = const_cast<double *>(base);
  GemmBatch p1, p2;
  int kmax = 1;
  for (size_t i = 0; i < n; ++i) {
    const ProductSlots sl{0, 0, 0, 0, trees[i]->arena - base, sig[i].X - base, sig[i].Y - base,
                          (P.w + w_base[i]) - base};
    append_product(p1, p2, *trees[i], op, sig[i].k, sig[i].ldx, sig[i].ldy, sl, w_off[i]);
    kmax = std::max(kmax, sig[i].k);
  }
  P.ph1 = tune_phase(p1, 1, op, kmax, P, s, autotune);
  P.ph2 = tune_phase(p2, 2, op, kmax, P, s, autotune);
}

}  // namespace

void batched_product(const std::vector<std::shared_ptr<DeviceTree>> &trees, ProdOp op,
                     Precision prec, const std::vector<const double *> &X,
                     const std::vector<int> &k, const std::vector<long long> &ldx,
                     const std::vector<double *> &Y, const std::vector<long long> &ldy,
                     cudaStream_t stream) {
  const size_t n = trees.size();
  HB_REQUIRE(X.size() == n && k.size() == n && ldx.size() == n && Y.size() == n &&
                 ldy.size() == n,
             INPUT_ERROR, "batched product: argument counts differ");
  if (n == 0) return;
  int device = 0;
  HB_CUDA(cudaGetDevice(&device));
  std::vector<BatchEntry> sig;
  for (size_t i = 0; i < n; ++i) {
    HB_REQUIRE(trees[i] != nullptr && X[i] != nullptr && Y[i] != nullptr, INPUT_ERROR,
               "batched product: NULL tree or buffer");
    HB_REQUIRE(trees[i]->device == device, INPUT_ERROR,
               "batched product: tree lives on another device");
    const long long rows = (op == ProdOp::L) ? k[i] : trees[i]->g.n;
    HB_REQUIRE(k[i] > 0 && ldx[i] >= std::max(1LL, rows) && ldy[i] >= std::max(1LL, rows),
               INPUT_ERROR, "batched product: leading dimension below the number of rows");
    HB_REQUIRE(((uintptr_t)X[i] | (uintptr_t)Y[i]) % sizeof(double) == 0, INPUT_ERROR,
               "batched product: buffers must be 8-byte aligned");
    sig.push_back(BatchEntry{trees[i], trees[i].get(), X[i], k[i], ldx[i], Y[i], ldy[i]});
  }
  if (prec == Precision::MIXED)
    HB_REQUIRE(op == ProdOp::N, INPUT_ERROR, "mixed precision is available for Y = H X (op N)");

  std::lock_guard<std::mutex> lk(g_batch_mutex);
  BatchPlan *P = nullptr;
  for (auto it = g_batch_cache.begin(); it != g_batch_cache.end(); ++it)
    if (same_signature(**it, (int)op, (int)prec, device, sig)) {
      g_batch_cache.splice(g_batch_cache.begin(), g_batch_cache, it);
      P = g_batch_cache.front().get();
      break;
    }
  const bool timing = option("record_phase_times", 0.0) != 0.0;
  if (!P) {
    auto plan = std::make_unique<BatchPlan>();
    plan->op = (int)op;
    plan->precision = (int)prec;
    plan->device = device;
    plan->sig = sig;
    const bool autotune = option("autotune", 1.0) != 0.0;
    cudaStream_t s = lib_stream();
    // the caller's work on `stream` (inputs, outputs) comes first
    cudaEvent_t ready;
    HB_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    HB_CUDA(cudaEventRecord(ready, stream));
    HB_CUDA(cudaStreamWaitEvent(s, ready, 0));
    cudaEventDestroy(ready);
    if (prec == Precision::MIXED) {
      std::vector<MixedItem> items;
      for (size_t i = 0; i < n; ++i)
        items.push_back(MixedItem{trees[i].get(), X[i], k[i], ldx[i], Y[i], ldy[i]});
      plan->mixed = mixed_batch_build(items, s);
      plan->tuned = "mixed: one launch per step";
    } else {
      build_fp64(*plan, trees, op, sig, s, autotune);
    }
    HB_CUDA(cudaStreamSynchronize(s));
    if (option("use_graphs", 1.0) != 0.0) {
      // one un-captured run first, so every kernel attribute is set
      plan->run(s);
      HB_CUDA(cudaStreamSynchronize(s));
      const long long before = launches();
      HB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      plan->run(s);
      HB_CUDA(cudaStreamEndCapture(s, &plan->graph));
      plan->graph_launches = launches() - before;
      count_launch(-plan->graph_launches);
      HB_CUDA(cudaGraphInstantiate(&plan->exec, plan->graph, 0));
    }
    g_last_tuned = plan->tuned;
    g_batch_cache.push_front(std::move(plan));
    while (g_batch_cache.size() > kBatchCacheSize) g_batch_cache.pop_back();
    P = g_batch_cache.front().get();
  }
  PhaseTimer timer(stream);
  if (P->exec && !timing) {
    HB_CUDA(cudaGraphLaunch(P->exec, stream));
    count_launch(P->graph_launches);
  } else {
    P->run(stream);
  }
  timer.mark(1);
  timer.mark(2);
  if (P->mixed && option("check_status", 0.0) != 0.0 && mixed_batch_status(*P->mixed, stream))
    throw Error{SVD_FAILURE, "a mixed-precision kernel gave up waiting on a barrier"};
}

int batched_status() {
  std::lock_guard<std::mutex> lk(g_batch_mutex);
  int worst = 0;
  for (auto &p : g_batch_cache)
    if (p->mixed) worst = std::max(worst, mixed_batch_status(*p->mixed, lib_stream()));
  return worst;
}

std::string batched_tuning() {
  std::lock_guard<std::mutex> lk(g_batch_mutex);
  return g_last_tuned;
}

void batched_release() {
  std::lock_guard<std::mutex> lk(g_batch_mutex);
  g_batch_cache.clear();
}

}  // namespace hb
