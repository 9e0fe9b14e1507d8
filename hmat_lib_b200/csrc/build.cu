// Dense -> HODLR construction (replaces hmat_lib src/constructors.c:629-704:
// copy_diagonal_blocks :212, compress_matrix :449, compress_off_diagonal
// :308, svd_double src/lapack_wrapper.c:8).
//
// Off-diagonal blocks of all levels are disjoint, so every block of every
// level is compressed in the same batched launches (the reference walks the
// levels bottom-up with one OpenMP task per block).  Two paths:
//
//  * exact: min(m, n) <= exact_max -> one-sided Jacobi SVD of the block;
//  * sketched: adaptive blocked randomized range finder.  Each round draws a
//    Gaussian test matrix Om, forms Y = A Om - Q (B Om) with one pass over
//    the block, orthonormalises Y panel by panel against the basis Q (block
//    classical Gram-Schmidt applied twice, then TSQR), and appends
//    B^T = A^T Q_new with a second pass.  The columns of B^T are in turn
//    orthonormalised into P with their coefficients collected in R_B, so
//    A ~ Q R_B^T P^T.  A round stops adding columns once the residual norm
//    estimated from the newest panel, ||(I - QQ^T) A Om_p||_F / sqrt(w),
//    falls below eta * tol * (a lower bound of sigma_0).  A Jacobi SVD of the
//    small R_B^T then gives the singular values; the rank follows hmat_lib's
//    relative rule and U = Q U_R Sigma, V = P V_R.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>

#include "bjacobi.h"
#include "build.h"
#include "jacobi.h"
#include "rank_mlp.h"
#include "sketch_mixed.h"
#include "tsqr.h"
#include "workload.h"

namespace hb {

namespace {

enum GB { kA = 0, kWork = 1, kArena = 2 };

template <class T>
T *upload_vec(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1), s));
  if (!v.empty())
    h2d_async(d, v.data(), sizeof(T) * v.size(), s);
  return d;
}

struct SketchBlock {
  int b;                 // index into the build's flattened block list
  int bid;               // block index in its own tree (names its random test matrices)
  int depth;
  long long lda;         // leading dimension of the block's input
  int m, n, cap;
  long long a_off;       // offset of the block in the input (base kA)
  long long q, bt, p, rb, om, t, c, rn;   // offsets in the work buffer
  int ell = 0;
  bool done = false;
  double sig_lb = 0.0;   // lower bound of sigma_0: largest row norm of B
  int last_pw = 0;
  int first_w = 0;       // width of the first round (predicted, or sketch_first)
  int pred = -1;         // predicted rank (-1: none)
  bool one_shot = false; // first round sized by the predictor, judged at tol
  bool fell_back = false;
  int mix = -1;          // index in the int8 sketch products (-1: FP64 GEMMs)
};

// Device memory free or held unused by the device's default stream-ordered
// pool (bytes).
double device_avail_bytes() {
  size_t free_b = 0, total_b = 0;
  HB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  double avail = (double)free_b;
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) ==
            cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used)
      avail += (double)(reserved - used);
  }
  (void)cudaGetLastError();
  return avail;
}

// Reads descs[i] (a column of up to `stride` doubles each, dst unused) into
// row i of `host` (rows of `stride` doubles): one gather launch into
// stream-ordered staging and one copy back instead of a copy per block.
// Synchronises with `s`.
void gather_to_host(std::vector<CopyDesc> descs, int stride, double *host, cudaStream_t s) {
  if (descs.empty()) return;
  const int nrow = (int)descs.size();
  double *stage = dev_alloc((size_t)nrow * stride, s);
  std::vector<CopyDesc> live;
  for (int i = 0; i < nrow; ++i) {
    CopyDesc &d = descs[i];
    if (d.rows <= 0) continue;
    d.dst = stage + (long long)i * stride;
    d.ldd = stride;
    d.cols = 1;
    live.push_back(d);
  }
  if (!live.empty()) {
    CopyDesc *dd = upload_vec(live, s);
    copy2d_batched(dd, (int)live.size(), s);
    cudaFreeAsync(dd, s);
  }
  HB_CUDA(cudaMemcpyAsync(host, stage, sizeof(double) * nrow * stride, cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  dev_free(stage, s);
}

thread_local BuildStats g_last_stats;
thread_local std::vector<float> g_last_features;

constexpr int kFeatCols = 16;   // width of the feature sketch

// Rank-model features of every sketched block (rank_mlp.h): a 16-column
// Gaussian sketch Y = A_b Omega, its R factor by TSQR and the singular values
// of R (= those of Y) by the batched Jacobi SVD, then log block size, depth,
// ln(kernel length) and five log ratios of the sketch's singular values.
std::vector<float> block_features(const std::vector<SketchBlock> &sk,
                                  const double *d_A, int aslot,
                                  const KernelSpec &gen, unsigned long long seed,
                                  cudaStream_t stream) {
  const int nsk = (int)sk.size();
  std::vector<float> f((size_t)nsk * kRankIn, 0.f);
  if (nsk == 0) return f;
  long long total = 0;
  constexpr int F = kFeatCols;
  std::vector<long long> om(nsk), y(nsk), r(nsk), ws(nsk), u(nsk), v(nsk), sg(nsk);
  auto take = [&](long long e) {
    const long long o = total;
    total += align_up(std::max<long long>(e, 1));
    return o;
  };
  for (int i = 0; i < nsk; ++i) {
    const SketchBlock &S = sk[i];
    om[i] = take((long long)S.n * F);
    y[i] = take((long long)S.m * F);
    r[i] = take(F * F);
    ws[i] = take(jacobi_workspace(F, F));
    u[i] = take(F * F);
    v[i] = take(F * F);
    sg[i] = take(F);
  }
  double *w = dev_alloc(total, stream);
  HB_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * total, stream));
  int *d_rank = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d_rank, sizeof(int) * (nsk + 1), stream));
  HB_CUDA(cudaMemsetAsync(d_rank, 0, sizeof(int) * (nsk + 1), stream));
  std::vector<RandDesc> rd;
  for (int i = 0; i < nsk; ++i)
    rd.push_back(RandDesc{w + om[i], sk[i].n, sk[i].n, F,
                          (1ULL << 60) + ((unsigned long long)sk[i].bid << 8)});
  gaussian_fill(rd, seed, stream);
  GemmBases bases{};
  bases.p[0] = const_cast<double *>(d_A);
  for (int i = 1; i < kGemmBases; ++i) bases.p[i] = w;
  bases.gen = gen;
  GemmBatch gb;
  for (int i = 0; i < nsk; ++i) {
    const SketchBlock &S = sk[i];
    int pr = gb.add(1, y[i], S.m, S.m, F);
    gb.seg(pr, aslot, S.a_off, S.lda, 0, 1, om[i], S.n, 0, S.n);
  }
  gemm_f64_run(gb, bases, TileShape::M128N64, stream);
  std::vector<TsqrProb> tp;
  for (int i = 0; i < nsk; ++i) {
    TsqrProb t;
    t.Y = w + y[i];
    t.ldy = sk[i].m;
    t.m = sk[i].m;
    t.w = F;
    t.R = w + r[i];
    t.ldr = F;
    tp.push_back(t);
  }
  tsqr_batched(tp, stream);
  std::vector<JacobiProb> jp;
  for (int i = 0; i < nsk; ++i) {
    JacobiProb q{};
    q.A = w + r[i];
    q.lda = F;
    q.m = F;
    q.n = F;
    q.G = w + ws[i];
    q.W = q.G + align_up(F * F);
    q.U = w + u[i];
    q.ldu = F;
    q.V = w + v[i];
    q.ldv = F;
    q.sigma = w + sg[i];
    q.rank = d_rank + i;
    jp.push_back(q);
  }
  JacobiParams prm;
  prm.trunc = Truncation::None;
  prm.max_sweeps = 30;
  JacobiProb *d_jp = upload_vec(jp, stream);
  jacobi_svd_batched(d_jp, nsk, prm, d_rank + nsk, F, stream);
  std::vector<double> sig((size_t)nsk * F);
  {
    std::vector<CopyDesc> gd;
    for (int i = 0; i < nsk; ++i) gd.push_back(CopyDesc{w + sg[i], F, nullptr, 0, F, 1});
    gather_to_host(gd, F, sig.data(), stream);
  }
  cudaFreeAsync(d_jp, stream);
  cudaFreeAsync(d_rank, stream);
  dev_free(w, stream);
  // kernel length scale: option kernel_length, else (matrix-free build) the
  // length of the kernel being compressed, else unknown (feature 0)
  double length = option("kernel_length", 0.0);
  if (length <= 0.0 && aslot == (int)kGenSlot) length = gen.length;
  for (int i = 0; i < nsk; ++i) {
    const SketchBlock &S = sk[i];
    float *row = &f[(size_t)i * kRankIn];
    row[0] = (float)std::log2((double)std::min(S.m, S.n));
    row[1] = (float)S.depth;
    row[2] = length > 0.0 ? (float)std::log(length) : 0.f;
    const double *sv = &sig[(size_t)i * F];
    const int idx[5] = {1, 3, 7, 11, 15};   // s_2, s_4, s_8, s_12, s_16
    for (int q = 0; q < 5; ++q) {
      const double rr = sv[0] > 0.0 ? sv[idx[q]] / sv[0] : 0.0;
      row[3 + q] = (float)std::max(-20.0, rr > 0.0 ? std::log10(rr) : -20.0);
    }
  }
  return f;
}
}  // namespace

const BuildStats &last_build_stats() { return g_last_stats; }
const std::vector<float> &last_build_features() { return g_last_features; }

namespace {

// The build.  With sketch_cap 0 every sketched block starts with a modest
// width cap -- 256 columns (option sketch_start) or an eighth of its width, or
// twice its predicted one-shot width -- so that a build whose ranks are small never reserves (and
// maps) scratch for wide sketches; a block that fills it moves its sketch
// into scratch of twice the width while the device memory allows (grow())
// and carries on.
std::vector<std::shared_ptr<DeviceTree>> build_attempt(
    const std::vector<BuildInput> &in, double tol, cudaStream_t stream, int *svd_status,
    BuildStats *stats, const KernelSpec *gen, std::chrono::steady_clock::time_point t0) {
  HB_REQUIRE(!in.empty(), INPUT_ERROR, "build: no tree to build");
  HB_REQUIRE(!gen || in.size() == 1, INPUT_ERROR, "a matrix-free build takes one tree");
  *svd_status = SUCCESS;
  // Every off-diagonal block of every tree, flattened.  The inputs are
  // addressed as element offsets from the lowest input address, so one GEMM
  // launch can read blocks of all of them.
  std::vector<Geometry> gs;
  const double *d_A = nullptr;
  for (const BuildInput &x : in) {
    gs.push_back(x.g);
    if (x.A && (!d_A || x.A < d_A)) d_A = x.A;
  }
  struct Blk {
    int t, b;
    BlockDesc B;
    long long a0;    // first entry of the block: offset from d_A (or generated origin)
    long long lda;
  };
  std::vector<Blk> blk;
  for (int t = 0; t < (int)in.size(); ++t)
    for (int b = 0; b < gs[t].nblock(); ++b) {
      const BlockDesc &B = gs[t].blocks[b];
      const long long a0 = gen ? gen_offset(B.r0, B.c0)
                               : (long long)(in[t].A - d_A) + B.r0 + (long long)B.c0 * in[t].lda;
      blk.push_back(Blk{t, b, B, a0, in[t].lda});
    }
  const int nb = (int)blk.size();
  const int exact_max = (int)option("exact_max", 128);
  const int cap_opt = (int)option("sketch_cap", 0.0) / kPanel * kPanel;
  const int w_first = std::max(kPanel, (int)option("sketch_first", 64) / kPanel * kPanel);
  const int w_next = std::max(kPanel, (int)option("sketch_step", 64) / kPanel * kPanel);
  const double eta = option("sketch_eta", 0.01);
  const unsigned long long seed = (unsigned long long)option("sketch_seed", 20240607);
  // operand of the block reads: the dense input, or the generated kernel matrix
  const KernelSpec gspec = gen ? *gen : KernelSpec();
  const int aslot = gen ? (int)kGenSlot : (int)kA;

  // ---- partition the blocks --------------------------------------------------
  std::vector<int> exact, sketched;
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = blk[b].B;
    const int C = std::min(B.m, B.n);
    if (C == 0) continue;
    (C <= exact_max ? exact : sketched).push_back(b);
  }

  // ---- scratch layout ----------------------------------------------------------
  long long scratch = 0;
  auto take = [&](long long elems) {
    const long long o = scratch;
    scratch += align_up(std::max<long long>(elems, 1));
    return o;
  };
  struct ExactSlot { long long ws, u, v, sig; };
  std::vector<ExactSlot> eslots;
  int max_c = 0;
  for (int b : exact) {
    const BlockDesc &B = blk[b].B;
    const int C = std::min(B.m, B.n);
    ExactSlot s;
    s.ws = take(jacobi_workspace(B.m, B.n));
    s.u = take((long long)B.m * C);
    s.v = take((long long)B.n * C);
    s.sig = take(C);
    eslots.push_back(s);
    max_c = std::max(max_c, C);
  }
  // Option build_precision = 1 (dense input only): the sketch products
  // Y = A Omega and B^T = A^T Q on the int8 tensor cores, every block sliced
  // once here (before the sketch widths are sized, so the slices count
  // against the memory); blocks whose sizes are not multiples of 32 keep the
  // FP64 GEMMs.
  std::unique_ptr<SketchMixed> smix;
  std::vector<int> mix_of(sketched.size(), -1);
  if (!gen && option("build_precision", 0.0) == 1.0) {
    std::vector<SketchMixedBlock> mb;
    for (size_t si = 0; si < sketched.size(); ++si) {
      const Blk &X = blk[sketched[si]];
      if (X.B.m % 32 || X.B.n % 32) continue;
      mix_of[si] = (int)mb.size();
      mb.push_back(SketchMixedBlock{d_A + X.a0, X.lda, X.B.m, X.B.n});
    }
    if (!mb.empty()) smix = std::make_unique<SketchMixed>(mb, stream);
  }
  // Sketch width caps.  Option sketch_cap > 0 fixes one cap for every block;
  // 0 (default): a block may grow to its full width, as long as each growth
  // of its scratch (and the core SVD that will follow) fits option
  // sketch_mem_frac (default 0.6) of the device memory that is free or held
  // unused by the stream-ordered pool at that moment (see grow()).
  std::vector<int> caps(sketched.size(), 0);
  for (size_t i = 0; i < sketched.size(); ++i) {
    const BlockDesc &B = blk[sketched[i]].B;
    const int C = std::min(B.m, B.n);
    caps[i] = cap_opt > 0 ? std::min(C, std::max(cap_opt, kPanel)) : C;
  }
  std::vector<SketchBlock> sk;
  for (size_t si = 0; si < sketched.size(); ++si) {
    const int b = sketched[si];
    const BlockDesc &B = blk[b].B;
    SketchBlock S;
    S.b = b;
    S.bid = blk[b].b;
    S.depth = B.depth;
    S.lda = blk[b].lda;
    S.m = B.m;
    S.n = B.n;
    S.cap = caps[si];
    S.a_off = blk[b].a0;
    S.mix = mix_of[si];
    sk.push_back(S);
  }
  // ---- learned sizing of the first sketch ---------------------------------------------
  const bool learned = option("learned_ranks", 0.0) != 0.0;
  const bool record = learned || option("record_features", 0.0) != 0.0;
  std::vector<float> feats;
  std::vector<float> model;
  const bool have_model = learned && rank_model(model);
  for (SketchBlock &S : sk) S.first_w = std::min(w_first, S.cap);
  const auto tf0 = std::chrono::steady_clock::now();
  if (record && !sk.empty()) {
    feats = block_features(sk, d_A, aslot, gspec, seed, stream);
    if (have_model) {
      const int nsk = (int)sk.size();
      float *dbuf = nullptr;
      HB_CUDA(cudaMallocAsync((void **)&dbuf, sizeof(float) * (kRankParams + nsk * (kRankIn + 1)),
                              stream));
      HB_CUDA(cudaMemcpyAsync(dbuf, model.data(), sizeof(float) * kRankParams,
                              cudaMemcpyHostToDevice, stream));
      HB_CUDA(cudaMemcpyAsync(dbuf + kRankParams, feats.data(), sizeof(float) * nsk * kRankIn,
                              cudaMemcpyHostToDevice, stream));
      float *dout = dbuf + kRankParams + nsk * kRankIn;
      rank_mlp_predict(dbuf, dbuf + kRankParams, nsk, dout, stream);
      std::vector<float> pred(nsk);
      HB_CUDA(cudaMemcpyAsync(pred.data(), dout, sizeof(float) * nsk, cudaMemcpyDeviceToHost,
                              stream));
      HB_CUDA(cudaStreamSynchronize(stream));
      cudaFreeAsync(dbuf, stream);
      // one-shot width: the predicted rank plus a margin, whole panels
      const double rel = option("learned_margin", 0.1);
      const int add = (int)option("learned_extra", 40);
      for (int i = 0; i < nsk; ++i) {
        SketchBlock &S = sk[i];
        const double r = std::max(1.0, std::exp2((double)std::min(pred[i], 20.f)) - 1.0);
        S.pred = (int)std::lround(r);
        const int w = (int)std::ceil(r * (1.0 + rel)) + add;
        S.first_w = std::min(S.cap, std::max(kPanel, (w + kPanel - 1) / kPanel * kPanel));
        S.one_shot = true;
      }
    }
  }
  // starting caps: option sketch_start (256) columns, an eighth of the width
  // if that is more, or twice the one-shot width; grown on demand
  const int start_cap = std::max(2 * kPanel, (int)option("sketch_start", 256) / kPanel * kPanel);
  std::vector<int> memcap(sk.size());
  for (size_t i = 0; i < sk.size(); ++i) {
    SketchBlock &S = sk[i];
    memcap[i] = S.cap;
    if (cap_opt <= 0) {
      // blocks wider than 8 start_cap columns start at an eighth of their
      // width (a wide block's rank can reach thousands: fewer growths, each a
      // fresh allocation of several GB)
      const int base = std::max(start_cap, std::min(S.m, S.n) / 8 / kPanel * kPanel);
      const int want = std::max(base, (2 * S.first_w + kPanel - 1) / kPanel * kPanel);
      S.cap = std::min(S.cap, want);
    }
  }
  // scratch of the sketched blocks: test matrices and products as wide as a
  // block's widest round
  int w_max = std::max(w_first, w_next);
  for (SketchBlock &S : sk) {
    const int wb = std::max(S.first_w, w_next);
    w_max = std::max(w_max, wb);
    S.q = take((long long)S.m * S.cap);
    S.bt = take((long long)S.n * S.cap);
    S.p = take((long long)S.n * S.cap);
    S.rb = take((long long)S.cap * S.cap);
    S.om = take((long long)S.n * wb);
    S.t = take((long long)S.cap * wb);
    S.c = take((long long)S.cap * kPanel);
    S.rn = take((long long)kPanel * kPanel + kPanel + wb);
  }
  const double ms_features =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tf0).count();
  const double eta_learned = option("learned_eta", 1.0);

  double *work = dev_alloc(scratch, stream);
  GemmBases bases{};
  bases.p[kA] = const_cast<double *>(d_A);
  bases.gen = gspec;
  bases.p[kWork] = work;
  for (int i = 2; i < kGemmBases; ++i) bases.p[i] = work;
  if (!sk.empty()) HB_CUDA(cudaMemsetAsync(work, 0, scratch * sizeof(double), stream));
  // A block at its cap whose memory-bounded cap is larger: Q, B^T, P and R_B
  // (with its first ell columns) and the round buffers sized by the cap move
  // to a fresh allocation of twice the width, addressed by offsets from
  // `work` like the rest.
  std::vector<double *> grown;
  const double mem_frac = option("sketch_mem_frac", 0.6);
  double limited_avail = -1.0;   // device memory seen by the first growth that did not fit
  auto grow = [&](SketchBlock &S, int limit) {
    const long long wbw = std::max(S.first_w, w_next);
    const long long m = S.m, n = S.n, e = S.ell;
    auto layout = [&](int c2, long long *parts) {
      parts[0] = align_up(m * c2);
      parts[1] = align_up(n * c2);
      parts[2] = align_up((long long)c2 * c2);
      parts[3] = align_up(c2 * wbw);
      parts[4] = align_up((long long)c2 * kPanel);
      return parts[0] + 2 * parts[1] + parts[2] + parts[3] + parts[4];
    };
    // twice the width, else smaller steps, whichever fits the memory budget
    // together with the block's core SVD (about five c2^2 doubles)
    const double avail = cap_opt > 0 ? 1e300 : device_avail_bytes();
    int c2 = 0;
    long long parts[5];
    for (int cand : {2 * S.cap, S.cap + S.cap / 2, S.cap + 256, S.cap + kPanel}) {
      const int c = std::min(limit, std::max(cand, S.cap + kPanel) / kPanel * kPanel);
      if (c <= S.cap) continue;
      if (8.0 * ((double)layout(c, parts) + 5.0 * (double)c * c) <= mem_frac * avail) {
        c2 = c;
        break;
      }
    }
    if (c2 == 0) {
      if (limited_avail < 0.0) limited_avail = avail;
      return;
    }
    const long long total = layout(c2, parts);
    const long long sq = parts[0], sb = parts[1], sr = parts[2], st = parts[3];
    double *g = dev_alloc(total, stream);
    grown.push_back(g);
    HB_CUDA(cudaMemsetAsync(g, 0, sizeof(double) * total, stream));
    const long long base = (long long)(g - work);
    const long long q = base, bt = q + sq, pp = bt + sb, rb = pp + sb, t = rb + sr, c = t + st;
    if (e > 0) {
      HB_CUDA(cudaMemcpyAsync(work + q, work + S.q, sizeof(double) * m * e,
                              cudaMemcpyDeviceToDevice, stream));
      HB_CUDA(cudaMemcpyAsync(work + bt, work + S.bt, sizeof(double) * n * e,
                              cudaMemcpyDeviceToDevice, stream));
      HB_CUDA(cudaMemcpyAsync(work + pp, work + S.p, sizeof(double) * n * e,
                              cudaMemcpyDeviceToDevice, stream));
      HB_CUDA(cudaMemcpy2DAsync(work + rb, sizeof(double) * c2, work + S.rb,
                                sizeof(double) * S.cap, sizeof(double) * e, (size_t)e,
                                cudaMemcpyDeviceToDevice, stream));
    }
    S.q = q;
    S.bt = bt;
    S.p = pp;
    S.rb = rb;
    S.t = t;
    S.c = c;
    S.cap = c2;
  };

  // ranks of exact blocks, ranks of sketched blocks, status, then the sweeps
  // used by every Jacobi problem in the same order
  int *d_int = nullptr;
  const int n_int = (int)exact.size() + (int)sk.size() + 1;
  HB_CUDA(cudaMallocAsync((void **)&d_int, sizeof(int) * 2 * n_int, stream));
  HB_CUDA(cudaMemsetAsync(d_int, 0, sizeof(int) * 2 * n_int, stream));
  int *d_status = d_int + n_int - 1;
  int *d_sweeps = d_int + n_int;
  JacobiParams prm;
  prm.tol = tol;
  prm.trunc = Truncation::Relative;
  prm.scale_u = 1;
  prm.max_sweeps = (int)option("jacobi_max_sweeps", 60);
  // option: a pair coupled at rounding level of the block's own norm counts as
  // orthogonal (moves no singular value by more than eps ||A||), fewer sweeps;
  // off by default: the normalised columns of the rotated side (hmat_lib's
  // orthonormal U or V) then keep couplings of up to eps ||A|| / sigma
  prm.norm_stop = option("jacobi_norm_stop", 0.0) != 0.0 ? 1 : 0;

  // stage events: start, exact done, rounds done, core SVDs done, end
  cudaEvent_t ev[5];
  for (auto &e : ev) HB_CUDA(cudaEventCreate(&e));
  HB_CUDA(cudaEventRecord(ev[0], stream));
  const double ms_setup =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

  // ---- exact path ----------------------------------------------------------------
  std::vector<JacobiProb> eprobs;
  for (size_t p = 0; p < exact.size(); ++p) {
    const BlockDesc &B = blk[exact[p]].B;
    const int R = std::max(B.m, B.n), C = std::min(B.m, B.n);
    JacobiProb jp{};
    if (gen) {
      jp.gen_r0 = B.r0;
      jp.gen_c0 = B.c0;
    } else {
      jp.A = d_A + blk[exact[p]].a0;
    }
    jp.lda = blk[exact[p]].lda;
    jp.transA = 0;
    jp.m = B.m;
    jp.n = B.n;
    jp.G = work + eslots[p].ws;
    jp.W = jp.G + align_up((long long)R * C);
    jp.U = work + eslots[p].u;
    jp.ldu = B.m;
    jp.V = work + eslots[p].v;
    jp.ldv = B.n;
    jp.sigma = work + eslots[p].sig;
    jp.rank = d_int + p;
    jp.sweeps = d_sweeps + p;
    eprobs.push_back(jp);
  }
  JacobiProb *d_eprobs = nullptr;
  if (!eprobs.empty()) {
    d_eprobs = upload_vec(eprobs, stream);
    jacobi_svd_batched(d_eprobs, (int)eprobs.size(), prm, d_status, max_c, stream, gspec);
  }

  HB_CUDA(cudaEventRecord(ev[1], stream));

  // ---- sketched path ---------------------------------------------------------------
  int rounds = 0;
  bool cap_hit = false;
  std::vector<double> host_rn;
  while (true) {
    std::vector<int> act;
    for (size_t i = 0; i < sk.size(); ++i)
      if (!sk[i].done) act.push_back((int)i);
    if (act.empty()) break;
    std::vector<int> wb(sk.size(), 0);
    for (int i : act) {
      const int wr = rounds == 0 ? sk[i].first_w : w_next;
      if (sk[i].ell >= sk[i].cap && sk[i].cap < memcap[i]) grow(sk[i], memcap[i]);
      wb[i] = std::min(wr, sk[i].cap - sk[i].ell);
      if (wb[i] <= 0) {
        sk[i].done = true;
        cap_hit = true;
      }
    }
    act.erase(std::remove_if(act.begin(), act.end(), [&](int i) { return wb[i] <= 0; }),
              act.end());
    if (act.empty()) break;

    // 1. Gaussian test matrices
    std::vector<RandDesc> rd;
    for (int i : act)
      rd.push_back(RandDesc{work + sk[i].om, sk[i].n, sk[i].n, wb[i],
                            ((unsigned long long)sk[i].bid << 24) + (unsigned long long)rounds});
    gaussian_fill(rd, seed, stream);

    // 2. Y = A Om written into the new columns of Q; 3. Y -= Q (B Om)
    {
      GemmBatch g1;
      std::vector<SketchMixed::Call> m1;
      for (int i : act) {
        const SketchBlock &S = sk[i];
        if (S.mix >= 0) {
          m1.push_back(SketchMixed::Call{S.mix, work + S.om, S.n, wb[i],
                                         work + S.q + (long long)S.ell * S.m, S.m});
          continue;
        }
        int pr = g1.add(kWork, S.q + (long long)S.ell * S.m, S.m, S.m, wb[i]);
        g1.seg(pr, aslot, S.a_off, S.lda, 0, kWork, S.om, S.n, 0, S.n);
      }
      gemm_f64_run(g1, bases, TileShape::M128N64, stream);
      if (smix) smix->multiply(false, m1, stream);
      // ||A om_c||^2: the scale against which a projected column counts as noise
      std::vector<NormDesc> nd;
      for (int i : act) {
        const SketchBlock &S = sk[i];
        nd.push_back(NormDesc{work + S.q + (long long)S.ell * S.m, S.m, S.m, wb[i],
                              work + S.rn + kPanel * kPanel + kPanel});
      }
      column_norms2(nd, stream);
      GemmBatch g2;
      for (int i : act) {
        const SketchBlock &S = sk[i];
        if (S.ell == 0) continue;
        int pr = g2.add(kWork, S.t, S.ell, S.ell, wb[i]);
        g2.seg(pr, kWork, S.bt, S.n, 1, kWork, S.om, S.n, 0, S.n);
      }
      gemm_f64_run(g2, bases, TileShape::M64N128, stream);
      GemmBatch g3;
      for (int i : act) {
        const SketchBlock &S = sk[i];
        if (S.ell == 0) continue;
        int pr = g3.add(kWork, S.q + (long long)S.ell * S.m, S.m, S.m, wb[i], -1.0, 1.0);
        g3.seg(pr, kWork, S.q, S.m, 0, kWork, S.t, S.ell, 0, S.ell);
      }
      gemm_f64_run(g3, bases, TileShape::M128N64, stream, false);
    }

    // 4. panel-wise orthonormalisation of the new Q columns (BCGS2 + TSQR)
    auto orthonormalise = [&](bool left) {
      int max_panels = 0;
      for (int i : act) max_panels = std::max(max_panels, (wb[i] + kPanel - 1) / kPanel);
      for (int q = 0; q < max_panels; ++q) {
        std::vector<int> pa;
        for (int i : act)
          if (q * kPanel < wb[i]) pa.push_back(i);
        for (int rep = 0; rep < 2; ++rep) {
          GemmBatch gc, gu;
          std::vector<CopyDesc> acc;
          for (int i : pa) {
            const SketchBlock &S = sk[i];
            const int p0 = S.ell + q * kPanel, pw = std::min(kPanel, wb[i] - q * kPanel);
            if (p0 == 0) continue;
            const int rows = left ? S.m : S.n;
            const long long base = left ? S.q : S.p;
            const long long panel = base + (long long)p0 * rows;
            // C (p0 x pw) = Base[:, :p0]^T Panel
            const long long cdst = left ? S.c : S.rb + (long long)p0 * S.cap;
            const long long cld = left ? S.cap : S.cap;
            const long long ctarget = (!left && rep == 0) ? cdst : S.c;
            int pr = gc.add(kWork, ctarget, left ? S.cap : cld, p0, pw);
            gc.seg(pr, kWork, base, rows, 1, kWork, panel, rows, 0, rows);
            // Panel -= Base[:, :p0] C
            int pu = gu.add(kWork, panel, rows, rows, pw, -1.0, 1.0);
            gu.seg(pu, kWork, base, rows, 0, kWork, ctarget, left ? S.cap : cld, 0, p0);
            if (!left && rep == 1)
              acc.push_back(CopyDesc{work + S.c, S.cap, work + cdst, S.cap, p0, pw});
          }
          gemm_f64_run(gc, bases, TileShape::M64N128, stream);
          gemm_f64_run(gu, bases, TileShape::M128N64, stream, false);
          if (!acc.empty()) {
            CopyDesc *d = upload_vec(acc, stream);
            add2d_batched(d, (int)acc.size(), 1.0, stream);
            cudaFreeAsync(d, stream);
          }
        }
        std::vector<TsqrProb> tp;
        for (int i : pa) {
          const SketchBlock &S = sk[i];
          const int p0 = S.ell + q * kPanel, pw = std::min(kPanel, wb[i] - q * kPanel);
          const int rows = left ? S.m : S.n;
          const long long base = left ? S.q : S.p;
          TsqrProb t;
          t.Y = work + base + (long long)p0 * rows;
          t.ldy = rows;
          t.m = rows;
          t.w = pw;
          if (left) {
            t.R = work + S.rn;
            t.ldr = kPanel;
          } else {
            t.R = work + S.rb + p0 + (long long)p0 * S.cap;
            t.ldr = S.cap;
          }
          tp.push_back(t);
          if (left) sk[i].last_pw = pw;
        }
        tsqr_batched(tp, stream);
        if (left) {
          std::vector<CleanDesc> cd;
          for (size_t a = 0; a < pa.size(); ++a) {
            const SketchBlock &S = sk[pa[a]];
            cd.push_back(CleanDesc{tp[a].Y, tp[a].ldy, tp[a].m, tp[a].w, tp[a].R, tp[a].ldr,
                                   work + S.rn + kPanel * kPanel + kPanel + q * kPanel});
          }
          panel_clean(cd, option("sketch_clean_rel", 1e-13), stream);
        }
      }
    };
    orthonormalise(true);

    // residual estimate of the last panel: ||R_last||_F^2
    {
      std::vector<NormDesc> nd;
      for (int i : act)
        nd.push_back(NormDesc{work + sk[i].rn, kPanel, sk[i].last_pw, sk[i].last_pw,
                              work + sk[i].rn + kPanel * kPanel});
      column_norms2(nd, stream);
    }

    // 5. B^T new columns = A^T Q_new; copy them to P for orthonormalisation
    {
      GemmBatch g5;
      std::vector<SketchMixed::Call> m5;
      for (int i : act) {
        const SketchBlock &S = sk[i];
        if (S.mix >= 0) {
          m5.push_back(SketchMixed::Call{S.mix, work + S.q + (long long)S.ell * S.m, S.m, wb[i],
                                         work + S.bt + (long long)S.ell * S.n, S.n});
          continue;
        }
        int pr = g5.add(kWork, S.bt + (long long)S.ell * S.n, S.n, S.n, wb[i]);
        g5.seg(pr, aslot, S.a_off, S.lda, 1, kWork, S.q + (long long)S.ell * S.m, S.m, 0, S.m);
      }
      gemm_f64_run(g5, bases, TileShape::M128N64, stream);
      if (smix) smix->multiply(true, m5, stream);
      std::vector<CopyDesc> cp;
      for (int i : act) {
        const SketchBlock &S = sk[i];
        cp.push_back(CopyDesc{work + S.bt + (long long)S.ell * S.n, S.n,
                              work + S.p + (long long)S.ell * S.n, S.n, S.n, wb[i]});
      }
      CopyDesc *d = upload_vec(cp, stream);
      copy2d_batched(d, (int)cp.size(), stream);
      cudaFreeAsync(d, stream);
    }
    // 6. P / R_B update
    orthonormalise(false);

    // 7. row norms of the new rows of B (= column norms of B^T)
    {
      std::vector<NormDesc> nd;
      for (int i : act) {
        const SketchBlock &S = sk[i];
        nd.push_back(NormDesc{work + S.bt + (long long)S.ell * S.n, S.n, S.n, wb[i],
                              work + S.t});
      }
      column_norms2(nd, stream);
    }
    // 8. read back and decide
    // per active block: its row norms of B (wb values, row 2a) and its last
    // panel's residual column norms (last_pw values, row 2a + 1), gathered and
    // read back in one copy
    std::vector<double> bn(act.size() * w_max, 0.0), rcols(act.size() * kPanel, 0.0);
    {
      const int stride = std::max(w_max, kPanel);
      std::vector<CopyDesc> gd;
      for (size_t a = 0; a < act.size(); ++a) {
        const SketchBlock &S = sk[act[a]];
        gd.push_back(CopyDesc{work + S.t, (long long)std::max(wb[act[a]], 1), nullptr, 0,
                              wb[act[a]], 1});
        gd.push_back(CopyDesc{work + S.rn + kPanel * kPanel, kPanel, nullptr, 0, S.last_pw, 1});
      }
      std::vector<double> h(gd.size() * (size_t)stride, 0.0);
      gather_to_host(gd, stride, h.data(), stream);
      for (size_t a = 0; a < act.size(); ++a) {
        std::copy(h.begin() + (2 * a) * stride, h.begin() + (2 * a) * stride + wb[act[a]],
                  bn.begin() + a * w_max);
        std::copy(h.begin() + (2 * a + 1) * stride, h.begin() + (2 * a + 1) * stride + kPanel,
                  rcols.begin() + a * kPanel);
      }
    }
    for (size_t a = 0; a < act.size(); ++a) {
      SketchBlock &S = sk[act[a]];
      double f2 = 0.0;
      for (int c = 0; c < S.last_pw; ++c) f2 += rcols[a * kPanel + c];
      for (int c = 0; c < wb[act[a]]; ++c) S.sig_lb = std::max(S.sig_lb, std::sqrt(bn[a * w_max + c]));
      S.ell += wb[act[a]];
      const double res = std::sqrt(f2 / std::max(S.last_pw, 1));
      // stop at the tolerance, or at the FP64 noise floor of the estimate; a
      // one-shot sketch sized by the predictor is accepted when the estimate
      // is within the tolerance itself, otherwise the block continues with
      // the plain adaptive rule
      const bool first_shot = S.one_shot && rounds == 0;
      const double floor_rel = std::max((first_shot ? eta_learned : eta) * tol, 1e-14);
      if (S.ell >= std::min(S.m, S.n) || S.sig_lb == 0.0 || res <= floor_rel * S.sig_lb)
        S.done = true;
      else if (first_shot)
        S.fell_back = true;
    }
    ++rounds;
  }

  HB_CUDA(cudaEventRecord(ev[2], stream));

  // ---- SVD of R_B^T for the sketched blocks ------------------------------------------
  // Cores of at least jacobi_block_min_c columns go to the block Jacobi solver
  // (one launch per round over the pairs of every core, on all SMs); the
  // others to the one-CTA / one-cluster solver.
  const int bj_min = (int)option("jacobi_block_min_c", 128);
  std::vector<JacobiProb> sprobs;
  std::vector<long long> s_u(sk.size()), s_v(sk.size());
  int max_l = 0;
  long long jscratch = 0;
  for (size_t i = 0; i < sk.size(); ++i) {
    const int L = sk[i].ell;
    const bool big = L >= bj_min;
    if (!big) max_l = std::max(max_l, L);
    jscratch += (big ? 0 : jacobi_workspace(L, L)) + 2 * align_up((long long)L * L) + align_up(L);
  }
  double *jwork = sk.empty() ? nullptr : dev_alloc(jscratch, stream);
  std::vector<char> is_big(sk.size(), 0);
  {
    long long o = 0;
    for (size_t i = 0; i < sk.size(); ++i) {
      const SketchBlock &S = sk[i];
      const int L = S.ell;
      is_big[i] = L >= bj_min;
      JacobiProb jp{};
      jp.A = work + S.rb;
      jp.lda = S.cap;
      jp.transA = 1;
      jp.m = L;
      jp.n = L;
      if (!is_big[i]) {
        jp.G = jwork + o;
        jp.W = jp.G + align_up((long long)L * L);
        o += jacobi_workspace(L, L);
      }
      jp.U = jwork + o;
      s_u[i] = o;
      jp.ldu = L;
      o += align_up((long long)L * L);
      jp.V = jwork + o;
      s_v[i] = o;
      jp.ldv = L;
      o += align_up((long long)L * L);
      jp.sigma = jwork + o;
      o += align_up(L);
      jp.rank = d_int + exact.size() + i;
      jp.sweeps = d_sweeps + exact.size() + i;
      sprobs.push_back(jp);
    }
  }
  JacobiProb *d_sprobs = nullptr;
  {
    std::vector<JacobiProb> small;
    std::vector<BjProb> big;
    for (size_t i = 0; i < sk.size(); ++i) {
      const JacobiProb &jp = sprobs[i];
      if (is_big[i])
        big.push_back(BjProb{jp.A, jp.lda, jp.m, jp.U, jp.V, jp.sigma, jp.rank, jp.sweeps});
      else
        small.push_back(jp);
    }
    if (!small.empty()) {
      d_sprobs = upload_vec(small, stream);
      jacobi_svd_batched(d_sprobs, (int)small.size(), prm, d_status, max_l, stream);
    }
    if (!big.empty()) block_jacobi_svd(big, tol, prm.max_sweeps, d_status, stream);
  }
  HB_CUDA(cudaEventRecord(ev[3], stream));
  std::vector<int> ints(2 * n_int, 0);
  HB_CUDA(cudaMemcpyAsync(ints.data(), d_int, sizeof(int) * 2 * n_int, cudaMemcpyDeviceToHost,
                          stream));
  // Frobenius epsilon-rank of every sketched block (for the rank model's
  // training data): the fewest leading singular values whose discarded tail
  // has Frobenius norm <= tol * s_0
  std::vector<int> fro_rank(sk.size(), 0);
  // (training data only: the singular values of every core come back to the
  // host, so a learned build without option record_features skips it)
  const bool want_fro = option("record_features", 0.0) != 0.0;
  std::vector<std::vector<double>> core_sig(want_fro ? sk.size() : 0);
  for (size_t i = 0; i < core_sig.size(); ++i) {
    core_sig[i].resize(sk[i].ell);
    HB_CUDA(cudaMemcpyAsync(core_sig[i].data(), sprobs[i].sigma, sizeof(double) * sk[i].ell,
                            cudaMemcpyDeviceToHost, stream));
  }
  HB_CUDA(cudaStreamSynchronize(stream));
  for (size_t i = 0; i < core_sig.size(); ++i) {
    const std::vector<double> &sv = core_sig[i];
    if (sv.empty() || !(sv[0] > 0.0)) continue;
    double tail = 0.0;
    int r = (int)sv.size();
    const double lim = tol * sv[0];
    while (r > 1 && std::sqrt(tail + sv[r - 1] * sv[r - 1]) <= lim) {
      tail += sv[r - 1] * sv[r - 1];
      --r;
    }
    fro_rank[i] = r;
  }
  *svd_status = ints[n_int - 1];
  for (Geometry &g : gs)
    for (auto &B : g.blocks) B.s = 0;
  for (size_t p = 0; p < exact.size(); ++p)
    gs[blk[exact[p]].t].blocks[blk[exact[p]].b].s = ints[p];
  for (size_t i = 0; i < sk.size(); ++i)
    gs[blk[sk[i].b].t].blocks[blk[sk[i].b].b].s = ints[exact.size() + i];

  // ---- arenas: leaves from the input, factors from the scratch ------------------------
  std::vector<std::shared_ptr<DeviceTree>> dts;
  for (const Geometry &g : gs) dts.push_back(dtree_create(g, stream));
  std::vector<CopyDesc> copies;
  std::vector<GenBlock> gen_leaves;
  for (size_t t = 0; t < dts.size(); ++t) {
    const DeviceTree &dt = *dts[t];
    for (int i = 0; i < dt.g.nleaf(); ++i) {
      const LeafDesc &L = dt.leaves[i];
      if (L.m == 0) continue;
      if (gen)
        gen_leaves.push_back(GenBlock{L.r0, L.r0, L.m, L.m, dt.arena + L.off, L.m});
      else
        copies.push_back(CopyDesc{in[t].A + L.r0 + (long long)L.r0 * in[t].lda, in[t].lda,
                                  dt.arena + L.off, L.m, L.m, L.m});
    }
  }
  kernel_blocks(gspec, gen_leaves, stream);
  for (size_t p = 0; p < exact.size(); ++p) {
    const DeviceTree &dt = *dts[blk[exact[p]].t];
    const BlockDesc &B = dt.g.blocks[blk[exact[p]].b];
    if (B.s == 0) continue;
    copies.push_back(CopyDesc{eprobs[p].U, B.m, dt.arena + B.u_off, B.m, B.m, B.s});
    copies.push_back(CopyDesc{eprobs[p].V, B.n, dt.arena + B.v_off, B.n, B.n, B.s});
  }
  if (!copies.empty()) {
    CopyDesc *d = upload_vec(copies, stream);
    copy2d_batched(d, (int)copies.size(), stream);
    cudaFreeAsync(d, stream);
  }
  if (!sk.empty()) {
    // U = Q[:, :ell] (U_R Sigma)[:, :s],  V = P[:, :ell] V_R[:, :s]; the arenas
    // are addressed from the lowest arena address
    double *abase = dts[0]->arena;
    for (auto &dt : dts) abase = std::min(abase, dt->arena);
    GemmBases fb{};
    fb.p[0] = work;
    fb.p[1] = jwork;
    fb.p[2] = abase;
    for (int i = 3; i < kGemmBases; ++i) fb.p[i] = work;
    GemmBatch gf;
    for (size_t i = 0; i < sk.size(); ++i) {
      const SketchBlock &S = sk[i];
      const DeviceTree &dt = *dts[blk[S.b].t];
      const BlockDesc &B = dt.g.blocks[blk[S.b].b];
      if (B.s == 0) continue;
      const long long ao = (long long)(dt.arena - abase);
      int pu = gf.add(2, ao + B.u_off, B.m, B.m, B.s);
      gf.seg(pu, 0, S.q, S.m, 0, 1, s_u[i], S.ell, 0, S.ell);
      int pv = gf.add(2, ao + B.v_off, B.n, B.n, B.s);
      gf.seg(pv, 0, S.p, S.n, 0, 1, s_v[i], S.ell, 0, S.ell);
    }
    gemm_f64_run(gf, fb, TileShape::M128N64, stream, false);
  }
  HB_CUDA(cudaEventRecord(ev[4], stream));
  HB_CUDA(cudaStreamSynchronize(stream));
  float stage_ms[4] = {0.f, 0.f, 0.f, 0.f};
  for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
  for (auto &e : ev) cudaEventDestroy(e);
  dev_free(d_eprobs, stream);
  dev_free(d_sprobs, stream);
  dev_free(d_int, stream);
  dev_free(jwork, stream);
  dev_free(work, stream);
  for (double *g : grown) dev_free(g, stream);
  HB_CUDA(cudaStreamSynchronize(stream));
  if (smix && smix->status(stream) != SUCCESS) {
    *svd_status = SVD_FAILURE;
    set_last_error("an int8 sketch product gave up waiting on a barrier");
  }
  smix.reset();
  if (cap_hit) {
    *svd_status = SVD_FAILURE;
    set_last_error(cap_opt > 0
                       ? "a block's rank reached the sketch cap (option sketch_cap)"
                       : "a block's rank reached the sketch width that fits the device memory "
                         "(option sketch_mem_frac; " +
                             std::to_string((long long)(limited_avail / 1e9)) +
                             " GB free or unused in the pool when it could not grow)");
  }
  BuildStats st;
  st.exact_blocks = (int)exact.size();
  st.sketched_blocks = (int)sk.size();
  st.sketch_rounds = rounds;
  st.cap_hit = cap_hit ? 1 : 0;
  const int maxsw = prm.max_sweeps;
  for (size_t p = 0; p < exact.size(); ++p) {
    const int sw = ints[n_int + p];
    st.max_sweeps_exact = std::max(st.max_sweeps_exact, sw);
    st.failed_exact += sw > maxsw;
  }
  for (size_t i = 0; i < sk.size(); ++i) {
    const int sw = ints[n_int + exact.size() + i];
    st.max_sweeps_sketch = std::max(st.max_sweeps_sketch, sw);
    st.failed_sketch += sw > maxsw;
    st.max_sketch = std::max(st.max_sketch, sk[i].ell);
  }
  g_last_features.clear();
  if (record) {
    for (size_t i = 0; i < sk.size(); ++i) {
      for (int q = 0; q < kRankIn; ++q) g_last_features.push_back(feats[i * kRankIn + q]);
      g_last_features.push_back((float)ints[exact.size() + i]);
      g_last_features.push_back((float)sk[i].pred);
      g_last_features.push_back((float)sk[i].first_w);
      g_last_features.push_back(sk[i].fell_back ? 1.f : 0.f);
      g_last_features.push_back((float)sk[i].ell);
      g_last_features.push_back((float)fro_rank[i]);
      st.learned_fallbacks += sk[i].fell_back;
    }
  }
  st.ms_features = ms_features;
  st.gemm_flops = gemm_flops_counter();
  for (const Geometry &g : gs) st.input_elems += (double)g.n * g.n;
  st.ms_exact = stage_ms[0];
  st.ms_rounds = stage_ms[1];
  st.ms_core_svd = stage_ms[2];
  st.ms_finish = stage_ms[3];
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  st.ms_host_setup = ms_setup;
  st.ms_host_total = 1e3 * st.seconds;
  st.ms_host_plans = plan_host_ms();
  g_last_stats = st;
  if (stats) *stats = st;
  return dts;
}

}  // namespace

std::vector<std::shared_ptr<DeviceTree>> build_batch(const std::vector<BuildInput> &in,
                                                     double tol, cudaStream_t stream,
                                                     int *svd_status, BuildStats *stats,
                                                     const KernelSpec *gen) {
  const auto t0 = std::chrono::steady_clock::now();
  gemm_flops_counter() = 0.0;
  plan_host_ms() = 0.0;
  return build_attempt(in, tol, stream, svd_status, stats, gen, t0);
}

std::shared_ptr<DeviceTree> build_from_dense(const Geometry &g, const double *d_A, long long lda,
                                             double tol, cudaStream_t stream, int *svd_status,
                                             BuildStats *stats, const KernelSpec *gen) {
  return build_batch({BuildInput{g, d_A, lda}}, tol, stream, svd_status, stats, gen)[0];
}

}  // namespace hb
