// Mixed-precision HODLR x dense product (op N) on the int8 tensor cores.
//
// Same two phases as the FP64 product (products.cu) with every GEMM done by
// the sliced int8 kernel (ozaki.cu):
//   1. W_b = V_b^T X_b for every block: A = V_b^T (rows = columns of V_b,
//      scaled per column), B = X (scaled per column over all rows), split
//      along n_b, partial tiles added atomically in FP64;
//   2. Y[leaf] = D X[leaf] + sum_levels U_b[rows] W_b: one tile per leaf band
//      and 64 columns, one K segment per term with its own scaling (D rows,
//      U_b rows, X columns, W_b columns per block).
// The slices of the tree's factors are made once and kept on the device;
// X and W are sliced at every call.  Requires leaf sizes that are multiples
// of 32 (16-byte aligned operand rows).
#include <algorithm>

#include "ozaki.h"
#include "products.h"

namespace hb {

struct MixedState {
  int8_t *bytes = nullptr;
  int *exps = nullptr;
  std::vector<long long> d_off, u_off, v_off;   // byte offsets of slice 0
  std::vector<long long> d_exp, u_exp, v_exp;   // int offsets
  std::vector<int> kpad, spad;
  std::map<std::pair<int, long long>, std::unique_ptr<struct MixedPlan>> plans;
  ~MixedState();
};

struct MixedPlan {
  int k = 0;
  int8_t *xs = nullptr;      // X slices [S][k][n]
  int *xe = nullptr;         // X column exponents [k]
  double *w = nullptr;       // W (FP64)
  int8_t *ws = nullptr;      // W slices, per block [S][k][spad_b]
  int *we = nullptr;         // W exponents, per block [k]
  std::vector<long long> w_off, ws_off, we_off;
  OzSeg *seg1 = nullptr, *seg2 = nullptr;
  OzTile *tile1 = nullptr, *tile2 = nullptr;
  int ntile1 = 0, ntile2 = 0;
  int *status = nullptr;
  std::vector<SliceJob> wjobs;
  ~MixedPlan() {
    for (void *p : {(void *)xs, (void *)xe, (void *)w, (void *)ws, (void *)we, (void *)seg1,
                    (void *)seg2, (void *)tile1, (void *)tile2, (void *)status})
      if (p) cudaFree(p);
  }
};

MixedState::~MixedState() {
  plans.clear();
  if (bytes) cudaFree(bytes);
  if (exps) cudaFree(exps);
}

namespace {

long long pad16(long long x) { return (x + 15) / 16 * 16; }
int pad32(int x) { return (x + 31) / 32 * 32; }

template <class T>
T *upload(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMalloc((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1)));
  if (!v.empty())
    HB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  return d;
}

MixedState &mixed_state(DeviceTree &t, cudaStream_t s) {
  if (t.mixed) return *t.mixed;
  const Geometry &g = t.g;
  for (int m : g.leaf_m)
    HB_REQUIRE(m % 32 == 0, INPUT_ERROR,
               "mixed precision needs leaf sizes that are multiples of 32");
  auto st = std::make_shared<MixedState>();
  const int S = kOzSlices;
  long long bytes = 0, ints = 0;
  const int nl = g.nleaf(), nb = g.nblock();
  st->d_off.resize(nl);
  st->d_exp.resize(nl);
  st->kpad.resize(nl);
  for (int i = 0; i < nl; ++i) {
    const int m = g.leaf_m[i];
    st->kpad[i] = pad32(m);
    st->d_off[i] = bytes;
    bytes += pad16((long long)S * m * st->kpad[i]);
    st->d_exp[i] = ints;
    ints += m;
  }
  st->u_off.resize(nb);
  st->v_off.resize(nb);
  st->u_exp.resize(nb);
  st->v_exp.resize(nb);
  st->spad.resize(nb);
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    st->spad[b] = pad32(std::max(B.s, 1));
    st->u_off[b] = bytes;
    bytes += pad16((long long)S * B.m * st->spad[b]);
    st->v_off[b] = bytes;
    bytes += pad16((long long)S * B.s * pad32(B.n));
    st->u_exp[b] = ints;
    ints += B.m;
    st->v_exp[b] = ints;
    ints += B.s;
  }
  HB_CUDA(cudaMalloc((void **)&st->bytes, std::max<long long>(bytes, 16)));
  HB_CUDA(cudaMalloc((void **)&st->exps, sizeof(int) * std::max<long long>(ints, 1)));
  HB_CUDA(cudaMemsetAsync(st->bytes, 0, std::max<long long>(bytes, 16), s));
  std::vector<SliceJob> jobs;
  for (int i = 0; i < nl; ++i) {
    const int m = g.leaf_m[i];
    if (m == 0) continue;
    jobs.push_back(SliceJob{t.arena + t.leaves[i].off, m, m, m, st->bytes + st->d_off[i],
                            (long long)m * st->kpad[i], st->kpad[i], st->exps + st->d_exp[i], 1});
  }
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (B.s == 0) continue;
    jobs.push_back(SliceJob{t.arena + B.u_off, B.m, B.m, B.s, st->bytes + st->u_off[b],
                            (long long)B.m * st->spad[b], st->spad[b], st->exps + st->u_exp[b], 1});
    jobs.push_back(SliceJob{t.arena + B.v_off, B.n, B.n, B.s, st->bytes + st->v_off[b],
                            (long long)B.s * pad32(B.n), pad32(B.n), st->exps + st->v_exp[b], 0});
  }
  ozaki_slice(jobs, s);
  HB_CUDA(cudaStreamSynchronize(s));
  t.mixed = st;
  return *st;
}

int covering(int h, int i, int d) {
  const int j = i >> (h - d);
  const bool top = ((i >> (h - d - 1)) & 1) == 0;
  return block_index(d, j, top ? 1 : 2);
}

MixedPlan &mixed_plan(DeviceTree &t, MixedState &st, int k, long long ldy, cudaStream_t s) {
  auto it = st.plans.find({k, ldy});
  if (it != st.plans.end()) return *it->second;
  const Geometry &g = t.g;
  const int S = kOzSlices, n = g.n, nb = g.nblock(), nl = g.nleaf(), h = g.h;
  const int npad = pad32(n);
  auto plan = std::make_unique<MixedPlan>();
  MixedPlan &P = *plan;
  P.k = k;
  const long long xslice = (long long)k * npad;
  HB_CUDA(cudaMalloc((void **)&P.xs, std::max<long long>(S * xslice, 16)));
  HB_CUDA(cudaMalloc((void **)&P.xe, sizeof(int) * std::max(k, 1)));
  long long wd = 0, wb = 0, we = 0;
  P.w_off.resize(nb);
  P.ws_off.resize(nb);
  P.we_off.resize(nb);
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    P.w_off[b] = wd;
    wd += align_up((long long)B.s * k);
    P.ws_off[b] = wb;
    wb += pad16((long long)S * k * st.spad[b]);
    P.we_off[b] = we;
    we += k;
  }
  HB_CUDA(cudaMalloc((void **)&P.w, sizeof(double) * std::max<long long>(wd, 1)));
  HB_CUDA(cudaMalloc((void **)&P.ws, std::max<long long>(wb, 16)));
  HB_CUDA(cudaMemsetAsync(P.ws, 0, std::max<long long>(wb, 16), s));
  HB_CUDA(cudaMalloc((void **)&P.we, sizeof(int) * std::max<long long>(we, 1)));
  HB_CUDA(cudaMalloc((void **)&P.status, sizeof(int)));
  HB_CUDA(cudaMemsetAsync(P.status, 0, sizeof(int), s));
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (B.s == 0) continue;
    P.wjobs.push_back(SliceJob{P.w + P.w_off[b], B.s, B.s, k, P.ws + P.ws_off[b],
                               (long long)k * st.spad[b], st.spad[b], P.we + P.we_off[b], 0});
  }
  // phase 1 tiles
  std::vector<OzSeg> s1;
  std::vector<OzTile> t1;
  const int kchunk_max = 2048;
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (B.s == 0) continue;
    const int nchunks = std::max(1, (B.n + kchunk_max - 1) / kchunk_max);
    const int chunk = pad32((B.n + nchunks - 1) / nchunks);
    for (int m0 = 0; m0 < B.s; m0 += kOzM)
      for (int n0 = 0; n0 < k; n0 += kOzN)
        for (int k0 = 0; k0 < B.n; k0 += chunk) {
          OzSeg sg;
          sg.a = OzOperand{st.bytes + st.v_off[b] + (long long)m0 * pad32(B.n) + k0,
                           (long long)B.s * pad32(B.n), pad32(B.n), st.exps + st.v_exp[b] + m0};
          sg.b = OzOperand{P.xs + (long long)n0 * npad + B.c0 + k0, xslice, npad, P.xe + n0};
          sg.K = std::min(chunk, B.n - k0);
          OzTile tl;
          tl.seg0 = (int)s1.size();
          tl.nseg = 1;
          tl.rows = std::min(kOzM, B.s - m0);
          tl.cols = std::min(kOzN, k - n0);
          tl.c_off = P.w_off[b] + m0 + (long long)n0 * B.s;
          tl.ldc = B.s;
          tl.atomic = 1;
          s1.push_back(sg);
          t1.push_back(tl);
        }
  }
  std::stable_sort(t1.begin(), t1.end(), [&](const OzTile &a, const OzTile &b) {
    return s1[a.seg0].K > s1[b.seg0].K;
  });
  // phase 2 tiles
  std::vector<OzSeg> s2;
  std::vector<OzTile> t2;
  for (int i = 0; i < nl; ++i) {
    const LeafDesc &L = t.leaves[i];
    for (int m0 = 0; m0 < L.m; m0 += kOzM)
      for (int n0 = 0; n0 < k; n0 += kOzN) {
        OzTile tl;
        tl.seg0 = (int)s2.size();
        tl.nseg = 0;
        tl.rows = std::min(kOzM, L.m - m0);
        tl.cols = std::min(kOzN, k - n0);
        tl.c_off = L.r0 + m0 + (long long)n0 * ldy;
        tl.ldc = ldy;
        tl.atomic = 0;
        OzSeg sd;
        sd.a = OzOperand{st.bytes + st.d_off[i] + (long long)m0 * st.kpad[i],
                         (long long)L.m * st.kpad[i], st.kpad[i], st.exps + st.d_exp[i] + m0};
        sd.b = OzOperand{P.xs + (long long)n0 * npad + L.r0, xslice, npad, P.xe + n0};
        sd.K = st.kpad[i];
        s2.push_back(sd);
        ++tl.nseg;
        for (int d = h - 1; d >= 0; --d) {
          const int b = covering(h, i, d);
          const BlockDesc &B = g.blocks[b];
          if (B.s == 0) continue;
          const int roff = L.r0 + m0 - B.r0;
          OzSeg su;
          su.a = OzOperand{st.bytes + st.u_off[b] + (long long)roff * st.spad[b],
                           (long long)B.m * st.spad[b], st.spad[b], st.exps + st.u_exp[b] + roff};
          su.b = OzOperand{P.ws + P.ws_off[b] + (long long)n0 * st.spad[b],
                           (long long)k * st.spad[b], st.spad[b], P.we + P.we_off[b] + n0};
          su.K = st.spad[b];
          s2.push_back(su);
          ++tl.nseg;
        }
        t2.push_back(tl);
      }
  }
  P.seg1 = upload(s1, s);
  P.tile1 = upload(t1, s);
  P.ntile1 = (int)t1.size();
  P.seg2 = upload(s2, s);
  P.tile2 = upload(t2, s);
  P.ntile2 = (int)t2.size();
  HB_CUDA(cudaStreamSynchronize(s));
  auto &ref = *plan;
  st.plans[{k, ldy}] = std::move(plan);
  return ref;
}

}  // namespace

void product_mixed(DeviceTree &t, const double *X, int k, long long ldx, double *Y, long long ldy,
                   cudaStream_t s) {
  if (k <= 0 || t.g.n == 0) return;
  std::lock_guard<std::mutex> lk(t.plan_mutex);
  MixedState &st = mixed_state(t, s);
  MixedPlan &P = mixed_plan(t, st, k, ldy, s);
  const int n = t.g.n, npad = pad32(n);
  PhaseTimer timer(s);
  // 1. slice X (columns, over all rows)
  ozaki_slice({SliceJob{X, ldx, n, k, P.xs, (long long)k * npad, npad, P.xe, 0}}, s);
  // 2. W = V^T X (split K, atomics into zeroed W)
  long long wtot = 0;
  for (auto &B : t.g.blocks) wtot += align_up((long long)B.s * k);
  HB_CUDA(cudaMemsetAsync(P.w, 0, sizeof(double) * std::max<long long>(wtot, 1), s));
  ozaki_gemm(P.seg1, P.tile1, P.ntile1, P.w, P.status, s);
  timer.mark(1);
  // 3. slice W per block; 4. Y = D X + sum U W
  ozaki_slice(P.wjobs, s);
  ozaki_gemm(P.seg2, P.tile2, P.ntile2, Y, P.status, s);
  timer.mark(2);
}

int mixed_status(DeviceTree &t, cudaStream_t s) {
  if (!t.mixed) return 0;
  int worst = 0;
  for (auto &kv : t.mixed->plans) {
    int v = 0;
    HB_CUDA(cudaMemcpyAsync(&v, kv.second->status, sizeof(int), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    worst = std::max(worst, v);
    HB_CUDA(cudaMemsetAsync(kv.second->status, 0, sizeof(int), s));
  }
  return worst;
}

}  // namespace hb
