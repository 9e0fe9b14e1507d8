// Mixed-precision HODLR x dense products on the int8 tensor cores: op N
// directly, op T and op L through the transposed tree (product_mixed_op).
//
// The FP64 product's two phases (products.cu), each one launch of the
// sliced int8 kernel (ozaki.cu):
//   1. W_b^T = X_b^T V_b for every block b: A = X^T (128 columns of X per
//      tile, K = the block's rows of X), B = V_b (<= 64 columns per tile).
//      Long blocks are split along K and added atomically in FP64.
//   2. Y[band] = [D | U_{b_h-1}[band] | ... | U_{b_0}[band]] [X[band]; W_{b_h-1}; ...; W_{b_0}]
//      for every 128-row band of every leaf and 64 columns of Y: one
//      concatenated K range per tile, so the tile is recombined once.  Every
//      row of the concatenated A shares one exponent (largest |entry| of the
//      leaf row and of the U rows beside it), every column of the
//      concatenated B one exponent (largest |entry| of that column of X and
//      of all W_b).
// Tree slices (A of phase 2, B of phase 1) are made once per tree; X is
// sliced twice per call (with its own column exponents for phase 1, with
// the common ones for phase 2) and W once.  Leaf sizes must be multiples of
// 32 (whole K-blocks).
#include <algorithm>
#include <tuple>

#include "jacobi.h"
#include "ozaki.h"
#include "products.h"
#include "tsqr.h"

namespace hb {

namespace {

int pad16(int x) { return (x + 15) / 16 * 16; }
int pad32(int x) { return (x + 31) / 32 * 32; }
long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

template <class T>
T *upload(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMalloc((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1)));
  if (!v.empty())
    HB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  return d;
}

template <class T>
T *dalloc(long long count) {
  T *d = nullptr;
  HB_CUDA(cudaMalloc((void **)&d, sizeof(T) * std::max<long long>(count, 1)));
  return d;
}

// Block of level d whose rows hold leaf i.
int covering(int h, int i, int d) {
  const int j = i >> (h - d);
  const bool top = ((i >> (h - d - 1)) & 1) == 0;
  return block_index(d, j, top ? 1 : 2);
}

// Every byte a segment, slice job or output tile touches lies inside the
// buffer it belongs to (checked on the host when a plan is made).
bool inside(const void *p, long long bytes, const void *base, long long size) {
  auto *q = (const uint8_t *)p, *b = (const uint8_t *)base;
  return bytes >= 0 && q >= b && q + bytes <= b + size;
}

void check_slice(const SliceJob &j, const void *buf, long long size) {
  HB_REQUIRE(j.nkb > 0 && j.ntiles > 0, INPUT_ERROR, "mixed plan: empty slice job");
  const long long last = (long long)(j.ntiles - 1) * j.tile_stride +
                         oz_offset(j.R, kOzSlices - 1, j.R - 1, (j.kb0 + j.nkb) * kOzKBlock - 1);
  HB_REQUIRE(inside(j.dst, last + 1, buf, size), INPUT_ERROR,
             "mixed plan: slice job outside its buffer");
}

void check_seg(const OzSeg &g, int nw, const void *abuf, long long asize, const void *bbuf0,
               long long bsize0, const void *bbuf1, long long bsize1) {
  HB_REQUIRE(g.nkb > 0, INPUT_ERROR, "mixed plan: empty segment");
  HB_REQUIRE(inside(g.a, (long long)g.nkb * kOzABlock, abuf, asize), INPUT_ERROR,
             "mixed plan: A segment outside its buffer");
  const long long bb = (long long)g.nkb * oz_bblock(nw);
  HB_REQUIRE(inside(g.b, bb, bbuf0, bsize0) || inside(g.b, bb, bbuf1, bsize1), INPUT_ERROR,
             "mixed plan: B segment outside its buffer");
}

}  // namespace

struct MixedPlan;

struct MixedState {
  uint8_t *bytes = nullptr;                // phase-2 A bands, phase-1 B tiles
  long long nbytes = 0;
  int *exps = nullptr;                     // row exponents [n], V column exponents
  unsigned long long *maxabs = nullptr;    // same layout, largest |entry|
  std::vector<long long> band_off;         // per leaf: bytes of its first 128-row band
  std::vector<int> band_nkb;               // per leaf: K-blocks of its concatenated row
  std::vector<long long> vb_off;           // per block: bytes of its first B tile
  std::vector<int> nw, ntn;                // per block: B tile width, number of tiles
  std::vector<long long> gexp;             // per block: offset of its column exponents
  std::map<std::tuple<int, long long, long long, int>, std::unique_ptr<MixedPlan>> plans;
  ~MixedState();
};

struct MixedPlan {
  int k = 0, nw2 = 0;
  unsigned long long *xmax = nullptr, *fmax = nullptr;
  int *xexp = nullptr, *fexp = nullptr;
  uint8_t *xa = nullptr, *xb = nullptr, *wb = nullptr;
  double *w = nullptr;
  long long w_zero = 0;                    // leading doubles of w added to atomically
  MaxBatch max_x, max_wsplit;
  SliceBatch sl_xa, sl_xb, sl_wb;
  OzSeg *seg1 = nullptr, *seg2 = nullptr;
  OzTile *tile1 = nullptr, *tile2 = nullptr;
  int ntile1 = 0, ntile2 = 0;
  int *start1 = nullptr, *start2 = nullptr;   // per-CTA tile runs (ozaki_schedule)
  int grid1 = 0, grid2 = 0;
  int *status = nullptr;
  // host copies for batches (X jobs with src NULL; phase-1 tiles relative to
  // w, phase-2 tiles relative to Y)
  std::vector<OzSeg> hs1, hs2;
  std::vector<OzTile> ht1, ht2;
  std::vector<MaxJob> hmx, hmw;
  std::vector<SliceJob> hsx, hsxb, hsb;
  ~MixedPlan() {
    for (void *p : {(void *)xmax, (void *)fmax, (void *)xexp, (void *)fexp, (void *)xa, (void *)xb,
                    (void *)wb, (void *)w, (void *)max_x.d, (void *)max_wsplit.d, (void *)sl_xa.d,
                    (void *)sl_xb.d, (void *)sl_wb.d, (void *)seg1, (void *)seg2, (void *)tile1,
                    (void *)tile2, (void *)start1, (void *)start2, (void *)status})
      if (p) cudaFree(p);
  }
};

MixedState::~MixedState() {
  plans.clear();
  if (bytes) cudaFree(bytes);
  if (exps) cudaFree(exps);
  if (maxabs) cudaFree(maxabs);
}

namespace {

MixedState &mixed_state(DeviceTree &t, cudaStream_t s) {
  if (t.mixed) return *t.mixed;
  const Geometry &g = t.g;
  for (int m : g.leaf_m)
    HB_REQUIRE(m % 32 == 0, INPUT_ERROR,
               "mixed precision needs leaf sizes that are multiples of 32");
  auto st = std::make_shared<MixedState>();
  const int nl = g.nleaf(), nb = g.nblock(), h = g.h, n = g.n;
  long long bytes = 0, nexp = n;
  st->band_off.resize(nl);
  st->band_nkb.resize(nl);
  for (int i = 0; i < nl; ++i) {
    int K = g.leaf_m[i];
    for (int d = h - 1; d >= 0; --d) K += pad32(g.blocks[covering(h, i, d)].s);
    HB_REQUIRE(K <= kOzMaxK, INPUT_ERROR, "mixed precision: leaf row plus ranks above 65536");
    st->band_nkb[i] = K / kOzKBlock;
    st->band_off[i] = bytes;
    bytes += cdiv(g.leaf_m[i], kOzRowsA) * (long long)st->band_nkb[i] * kOzABlock;
  }
  st->vb_off.assign(nb, 0);
  st->nw.assign(nb, 0);
  st->ntn.assign(nb, 0);
  st->gexp.assign(nb, 0);
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (B.s == 0) continue;
    st->ntn[b] = (int)cdiv(B.s, kOzMaxNw);
    st->nw[b] = pad16((int)cdiv(B.s, st->ntn[b]));
    st->vb_off[b] = bytes;
    bytes += (long long)st->ntn[b] * (B.n / kOzKBlock) * oz_bblock(st->nw[b]);
    st->gexp[b] = nexp;
    nexp += B.s;
  }
  st->bytes = dalloc<uint8_t>(bytes);
  st->nbytes = bytes;
  st->exps = dalloc<int>(nexp);
  st->maxabs = dalloc<unsigned long long>(nexp);
  HB_CUDA(cudaMemsetAsync(st->maxabs, 0, sizeof(unsigned long long) * nexp, s));

  std::vector<MaxJob> mj;
  std::vector<SliceJob> sj, sv;   // line-contiguous (D, U) and K-contiguous (V) sources
  for (int i = 0; i < nl; ++i) {
    const LeafDesc &L = t.leaves[i];
    const int bands = (int)cdiv(L.m, kOzRowsA);
    const long long stride = (long long)st->band_nkb[i] * kOzABlock;
    const double *D = t.arena + L.off;
    mj.push_back(MaxJob{D, 1, L.m, L.m, L.m, st->maxabs + L.r0, 0});
    sj.push_back(SliceJob{D, 1, L.m, L.m, L.m, kOzRowsA, bands, 0, L.m / kOzKBlock,
                          st->bytes + st->band_off[i], stride, st->maxabs + L.r0,
                          st->exps + L.r0, 0});
    int kb = L.m / kOzKBlock;
    for (int d = h - 1; d >= 0; --d) {
      const BlockDesc &B = g.blocks[covering(h, i, d)];
      if (B.s == 0) continue;
      const double *U = t.arena + B.u_off + (L.r0 - B.r0);
      sj.push_back(SliceJob{U, 1, B.m, L.m, B.s, kOzRowsA, bands, kb, pad32(B.s) / kOzKBlock,
                            st->bytes + st->band_off[i], stride, st->maxabs + L.r0, nullptr,
                            0});
      kb += pad32(B.s) / kOzKBlock;
    }
  }
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (B.s == 0) continue;
    mj.push_back(MaxJob{t.arena + B.u_off, 1, B.m, B.m, B.s, st->maxabs + B.r0, 0});
    const double *V = t.arena + B.v_off;
    mj.push_back(MaxJob{V, B.n, 1, B.s, B.n, st->maxabs + st->gexp[b], 0});
    const int nkb = B.n / kOzKBlock;
    sv.push_back(SliceJob{V, B.n, 1, B.s, B.n, st->nw[b], st->ntn[b], 0, nkb,
                          st->bytes + st->vb_off[b], (long long)nkb * oz_bblock(st->nw[b]),
                          st->maxabs + st->gexp[b], st->exps + st->gexp[b], 0});
  }
  for (const SliceJob &j : sj) check_slice(j, st->bytes, bytes);
  for (const SliceJob &j : sv) check_slice(j, st->bytes, bytes);
  MaxBatch bm = ozaki_max_batch(mj, s);
  SliceBatch bs = ozaki_slice_batch(sj, s), bv = ozaki_slice_batch(sv, s);
  ozaki_max(bm, nullptr, s);
  ozaki_slice(bs, nullptr, s);
  ozaki_slice(bv, nullptr, s);
  HB_CUDA(cudaStreamSynchronize(s));
  for (void *p : {(void *)bm.d, (void *)bs.d, (void *)bv.d})
    if (p) cudaFree(p);
  t.mixed = st;
  return *st;
}

MixedPlan &mixed_plan(DeviceTree &t, MixedState &st, int k, long long ldx, long long ldy,
                      cudaStream_t s, int min_depth = 0) {
  auto key = std::make_tuple(k, ldx, ldy, min_depth);
  auto it = st.plans.find(key);
  if (it != st.plans.end()) return *it->second;
  const Geometry &g = t.g;
  const int n = g.n, nb = g.nblock(), nl = g.nleaf(), h = g.h;
  const int nkbn = n / kOzKBlock;
  // blocks that take part: nonzero rank, depth >= min_depth (a product of
  // the leaves and the deeper blocks only: the block-diagonal product of
  // the subtrees rooted at min_depth)
  auto inc = [&](int b) { return g.blocks[b].s > 0 && g.blocks[b].depth >= min_depth; };
  auto plan = std::make_unique<MixedPlan>();
  MixedPlan &P = *plan;
  P.k = k;
  P.nw2 = std::min(kOzMaxNw, pad16(k));
  const int nja = (int)cdiv(k, kOzRowsA), njb = (int)cdiv(k, P.nw2);
  P.xmax = dalloc<unsigned long long>(k);
  P.fmax = dalloc<unsigned long long>(k);
  P.xexp = dalloc<int>(k);
  P.fexp = dalloc<int>(k);
  const long long xa_size = (long long)nja * nkbn * kOzABlock;
  const long long xb_size = (long long)njb * nkbn * oz_bblock(P.nw2);
  P.xa = dalloc<uint8_t>(xa_size);
  P.xb = dalloc<uint8_t>(xb_size);
  P.status = dalloc<int>(1);
  HB_CUDA(cudaMemsetAsync(P.status, 0, sizeof(int), s));

  // ---- phase 1 tiles: split long blocks along K so the work spreads -------------
  long long work = 0;
  for (int b = 0; b < nb; ++b)
    if (inc(b)) work += (long long)st.ntn[b] * st.nw[b] * (g.blocks[b].n / kOzKBlock);
  work *= nja;
  // about `per_cta` tiles' worth of work per CTA (option ozaki_phase1_tiles_per_cta)
  const long long per_cta = std::max(1LL, (long long)option("ozaki_phase1_tiles_per_cta", 2.0));
  const long long target = std::max<long long>(work / (per_cta * num_sms()), 64LL * 16);
  std::vector<int> nch(nb, 1);
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (!inc(b)) continue;
    const int nkb = B.n / kOzKBlock;
    nch[b] = (int)std::max(1LL, std::min<long long>(nkb / 8, cdiv((long long)st.nw[b] * nkb, target)));
    nch[b] = (int)std::max<long long>(nch[b], cdiv(nkb, kOzMaxK / kOzKBlock));
  }
  // W^T per block (k x s_b, ld k); blocks split along K first so one memset zeroes them
  std::vector<long long> w_off(nb, 0);
  long long wd = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (int b = 0; b < nb; ++b) {
      const BlockDesc &B = g.blocks[b];
      if (!inc(b) || (nch[b] > 1) != (pass == 0)) continue;
      w_off[b] = wd;
      wd += align_up((long long)B.s * k);
      if (pass == 0) P.w_zero = wd;
    }
  P.w = dalloc<double>(wd);
  std::vector<OzSeg> s1;
  std::vector<OzTile> t1;
  std::vector<long long> work1;
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (!inc(b)) continue;
    const int nkb = B.n / kOzKBlock, nw = st.nw[b];
    const int per = (int)cdiv(nkb, nch[b]);
    for (int tn = 0; tn < st.ntn[b]; ++tn)
      for (int kb0 = 0; kb0 < nkb; kb0 += per)
        for (int ja = 0; ja < nja; ++ja) {
          const int len = std::min(per, nkb - kb0);
          OzSeg sg{P.xa + ((long long)ja * nkbn + B.c0 / kOzKBlock + kb0) * kOzABlock,
                   st.bytes + st.vb_off[b] + ((long long)tn * nkb + kb0) * oz_bblock(nw), len, 0};
          OzTile tl;
          tl.seg0 = (int)s1.size();
          tl.nseg = 1;
          tl.rows = std::min(kOzRowsA, k - ja * kOzRowsA);
          tl.cols = std::min(nw, B.s - tn * nw);
          tl.nw = nw;
          tl.atomic = nch[b] > 1;
          tl.c_off = w_off[b] + ja * kOzRowsA + (long long)tn * nw * k;
          tl.ldc = k;
          tl.rexp = P.xexp + ja * kOzRowsA;
          tl.cexp = st.exps + st.gexp[b] + tn * nw;
          tl.rmax = nch[b] > 1 ? nullptr : P.fmax + ja * kOzRowsA;
          s1.push_back(sg);
          t1.push_back(tl);
          work1.push_back((long long)len * nw);
        }
  }
  // longest tiles first (round-robin over the persistent grid)
  std::vector<int> order(t1.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return work1[a] > work1[b]; });
  std::vector<OzTile> t1s;
  for (int i : order) t1s.push_back(t1[i]);

  // ---- phase 2 tiles: band-major so a band's column tiles run together ----------
  std::vector<long long> wb_off(nb, 0);
  long long wbb = 0;
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (!inc(b)) continue;
    wb_off[b] = wbb;
    wbb += (long long)njb * (pad32(B.s) / kOzKBlock) * oz_bblock(P.nw2);
  }
  P.wb = dalloc<uint8_t>(wbb);
  std::vector<OzSeg> s2;
  std::vector<OzTile> t2;
  for (int i = 0; i < nl; ++i) {
    const LeafDesc &L = t.leaves[i];
    const long long stride = (long long)st.band_nkb[i] * kOzABlock;
    for (int m0 = 0, band = 0; m0 < L.m; m0 += kOzRowsA, ++band)
      for (int jb = 0; jb < njb; ++jb) {
        OzTile tl;
        tl.seg0 = (int)s2.size();
        tl.nseg = 0;
        tl.rows = std::min(kOzRowsA, L.m - m0);
        tl.cols = std::min(P.nw2, k - jb * P.nw2);
        tl.nw = P.nw2;
        tl.atomic = 0;
        tl.c_off = L.r0 + m0 + (long long)jb * P.nw2 * ldy;
        tl.ldc = ldy;
        tl.rexp = st.exps + L.r0 + m0;
        tl.cexp = P.fexp + jb * P.nw2;
        tl.rmax = nullptr;
        const uint8_t *a = st.bytes + st.band_off[i] + band * stride;
        const int nkd = L.m / kOzKBlock;
        s2.push_back(OzSeg{a, P.xb + ((long long)jb * nkbn + L.r0 / kOzKBlock) * oz_bblock(P.nw2),
                           nkd, 0});
        a += (long long)nkd * kOzABlock;
        ++tl.nseg;
        for (int d = h - 1; d >= 0; --d) {
          const int b = covering(h, i, d);
          const BlockDesc &B = g.blocks[b];
          if (!B.s) continue;
          const int nks = pad32(B.s) / kOzKBlock;
          if (B.depth >= min_depth) {
            s2.push_back(
                OzSeg{a, P.wb + wb_off[b] + (long long)jb * nks * oz_bblock(P.nw2), nks, 0});
            ++tl.nseg;
          }
          a += (long long)nks * kOzABlock;
        }
        t2.push_back(tl);
      }
  }

  // ---- exponent and slicing jobs --------------------------------------------------
  std::vector<MaxJob> mx{MaxJob{nullptr, ldx, 1, k, n, P.xmax, 0}};
  std::vector<MaxJob> mw;   // W of the blocks split along K (the others: phase-1 epilogue)
  std::vector<SliceJob> sx{SliceJob{nullptr, ldx, 1, k, n, kOzRowsA, nja, 0, nkbn, P.xa,
                                    (long long)nkbn * kOzABlock, P.xmax, P.xexp, 0}};
  std::vector<SliceJob> sxb{SliceJob{nullptr, ldx, 1, k, n, P.nw2, njb, 0, nkbn, P.xb,
                                     (long long)nkbn * oz_bblock(P.nw2), P.fmax, P.fexp, 0}};
  std::vector<SliceJob> sb;
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    if (!inc(b)) continue;
    const double *wt = P.w + w_off[b];
    if (nch[b] > 1) mw.push_back(MaxJob{wt, 1, k, k, B.s, P.fmax, 0});
    const int nks = pad32(B.s) / kOzKBlock;
    sb.push_back(SliceJob{wt, 1, k, k, B.s, P.nw2, njb, 0, nks, P.wb + wb_off[b],
                          (long long)nks * oz_bblock(P.nw2), P.fmax, nullptr, 0});
  }
  for (size_t i = 0; i < t1.size(); ++i) {
    const OzTile &tl = t1[i];
    check_seg(s1[tl.seg0], tl.nw, P.xa, xa_size, st.bytes, st.nbytes, nullptr, 0);
    HB_REQUIRE(tl.c_off >= 0 && tl.c_off + (tl.rows - 1) + (tl.cols - 1) * tl.ldc < wd,
               INPUT_ERROR, "mixed plan: phase-1 tile outside W");
  }
  for (const OzTile &tl : t2) {
    long long K = 0;
    for (int q = tl.seg0; q < tl.seg0 + tl.nseg; ++q) {
      check_seg(s2[q], tl.nw, st.bytes, st.nbytes, P.xb, xb_size, P.wb, wbb);
      K += (long long)s2[q].nkb * kOzKBlock;
    }
    HB_REQUIRE(K <= kOzMaxK, INPUT_ERROR, "mixed plan: tile K above 65536");
  }
  check_slice(sx[0], P.xa, xa_size);
  check_slice(sxb[0], P.xb, xb_size);
  for (const SliceJob &j : sb) check_slice(j, P.wb, wbb);
  P.max_x = ozaki_max_batch(mx, s);
  P.max_wsplit = ozaki_max_batch(mw, s);
  P.sl_xa = ozaki_slice_batch(sx, s);
  P.sl_xb = ozaki_slice_batch(sxb, s);
  P.sl_wb = ozaki_slice_batch(sb, s);
  P.hs1 = s1;
  P.hs2 = s2;
  P.ht1 = t1s;
  P.ht2 = t2;
  P.hmx = mx;
  P.hmw = mw;
  P.hsx = sx;
  P.hsxb = sxb;
  P.hsb = sb;
  P.grid1 = ozaki_grid((int)t1s.size());
  P.grid2 = ozaki_grid((int)t2.size());
  P.start1 = upload(ozaki_schedule(t1s, s1, P.grid1), s);
  P.start2 = upload(ozaki_schedule(t2, s2, P.grid2), s);
  P.seg1 = upload(s1, s);
  P.tile1 = upload(t1s, s);
  P.ntile1 = (int)t1s.size();
  P.seg2 = upload(s2, s);
  P.tile2 = upload(t2, s);
  P.ntile2 = (int)t2.size();
  HB_CUDA(cudaStreamSynchronize(s));
  auto &ref = *plan;
  st.plans[key] = std::move(plan);
  return ref;
}

}  // namespace

void product_mixed(DeviceTree &t, const double *X, int k, long long ldx, double *Y, long long ldy,
                   cudaStream_t s, int min_depth) {
  if (k <= 0 || t.g.n == 0) return;
  HB_REQUIRE(ldx >= t.g.n && ldy >= t.g.n, INPUT_ERROR, "leading dimension below n");
  std::lock_guard<std::mutex> lk(t.plan_mutex);
  MixedState &st = mixed_state(t, s);
  MixedPlan &P = mixed_plan(t, st, k, ldx, ldy, s, min_depth);
  PhaseTimer timer(s);
  // 1. exponents and slices of X for phase 1; W^T = X^T V per block (the
  //    epilogue also folds the column maxima of unsplit blocks into fmax)
  HB_CUDA(cudaMemsetAsync(P.xmax, 0, sizeof(unsigned long long) * k, s));
  ozaki_max(P.max_x, X, s);
  ozaki_slice(P.sl_xa, X, s);
  HB_CUDA(cudaMemcpyAsync(P.fmax, P.xmax, sizeof(unsigned long long) * k,
                          cudaMemcpyDeviceToDevice, s));
  if (P.w_zero) HB_CUDA(cudaMemsetAsync(P.w, 0, sizeof(double) * P.w_zero, s));
  timer.kernel(1, false);
  ozaki_gemm(P.seg1, P.tile1, P.start1, P.grid1, P.w, P.status, s);
  timer.kernel(1, true);
  timer.mark(1);
  // 2. common column exponents of X and W, their slices; Y band by band
  ozaki_max(P.max_wsplit, X, s);
  ozaki_slice(P.sl_xb, X, s);
  ozaki_slice(P.sl_wb, X, s);
  timer.kernel(2, false);
  ozaki_gemm(P.seg2, P.tile2, P.start2, P.grid2, Y, P.status, s);
  timer.kernel(2, true);
  timer.mark(2);
}

// ---- H^T X and X H -------------------------------------------------------------------

namespace {

constexpr int kTT = 32;   // transpose tile

// dst (cols x rows, ld ldd) = src^T, src rows x cols (ld lds); 32 x 32 tiles
// through shared memory (one padding column against bank conflicts).
__global__ void transpose_kernel(const double *__restrict__ src, long long lds, int rows, int cols,
                                 double *__restrict__ dst, long long ldd) {
  __shared__ double tile[kTT][kTT + 1];
  const int r0 = blockIdx.x * kTT, c0 = blockIdx.y * kTT;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8 threads
  for (int j = ty; j < kTT; j += 8) {
    const int r = r0 + tx, c = c0 + j;
    if (r < rows && c < cols) tile[j][tx] = src[r + (long long)c * lds];
  }
  __syncthreads();
  for (int j = ty; j < kTT; j += 8) {
    const int c = c0 + tx, r = r0 + j;   // dst element (c, r)
    if (r < rows && c < cols) dst[c + (long long)r * ldd] = tile[tx][j];
  }
}

void transpose(const double *src, long long lds, int rows, int cols, double *dst, long long ldd,
               cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  for (int c0 = 0; c0 < cols; c0 += 65535 * kTT) {
    const int cc = std::min(cols - c0, 65535 * kTT);
    dim3 grid((rows + kTT - 1) / kTT, (cc + kTT - 1) / kTT);
    transpose_kernel<<<grid, dim3(kTT, 8), 0, s>>>(src + (long long)c0 * lds, lds, rows, cc,
                                                  dst + c0, ldd);
    HB_LAUNCHED();
  }
}

// Columns j of a block's U and V scaled by a and 1 / a, a = (|V_j| / |U_j|)^(1/2),
// so both get the norm (|U_j| |V_j|)^(1/2): the product U V^T is unchanged.
struct BalanceDesc {
  double *U, *V;
  int m, n, s;
  const double *nu2, *nv2;   // squared column norms of U and V
};
__global__ void balance_kernel(const BalanceDesc *__restrict__ d) {
  const BalanceDesc B = d[blockIdx.y];
  for (int j = blockIdx.x; j < B.s; j += gridDim.x) {
    const double nu = B.nu2[j], nv = B.nv2[j];
    if (!(nu > 0.0) || !(nv > 0.0)) continue;
    const double a = sqrt(sqrt(nv / nu)), ia = 1.0 / a;
    for (int i = threadIdx.x; i < B.m; i += blockDim.x) B.U[i + (long long)j * B.m] *= a;
    for (int i = threadIdx.x; i < B.n; i += blockDim.x) B.V[i + (long long)j * B.n] *= ia;
  }
}

// H^T as a device tree of the same geometry: leaf i is D_i^T, block (d, j, c)
// is the transpose of block (d, j, 3 - c) (U and V swapped), so H^T X is an
// op-N product of this tree.  Its U (the old V, orthonormal columns) and V
// (the old U, scaled by the singular values) are rebalanced to equal column
// norms: the int8 rows of the product concatenate a leaf row with U rows and
// share one exponent, so U entries far below the leaf's would lose bits.
DeviceTree &transposed_tree(DeviceTree &t, cudaStream_t s) {
  if (t.transposed) return *t.transposed;
  Geometry gt = t.g;
  for (int b = 0; b < gt.nblock(); ++b) {
    const BlockDesc &o = t.g.blocks[b ^ 1];
    BlockDesc &B = gt.blocks[b];
    B.m = o.n;
    B.n = o.m;
    B.s = o.s;
  }
  std::shared_ptr<DeviceTree> tt = dtree_create(gt, s);
  for (int i = 0; i < gt.nleaf(); ++i) {
    const int m = t.leaves[i].m;
    transpose(t.arena + t.leaves[i].off, m, m, m, tt->arena + tt->leaves[i].off, m, s);
  }
  std::vector<CopyDesc> cp;
  for (int b = 0; b < gt.nblock(); ++b) {
    const BlockDesc &o = t.g.blocks[b ^ 1], &B = tt->g.blocks[b];
    if (B.s == 0) continue;
    cp.push_back(CopyDesc{t.arena + o.v_off, o.n, tt->arena + B.u_off, B.m, B.m, B.s});
    cp.push_back(CopyDesc{t.arena + o.u_off, o.m, tt->arena + B.v_off, B.n, B.n, B.s});
  }
  if (!cp.empty()) {
    CopyDesc *d = upload(cp, s);
    copy2d_batched(d, (int)cp.size(), s);
    // rebalance every block's columns
    long long tot = 0;
    std::vector<long long> off(gt.nblock(), 0);
    for (int b = 0; b < gt.nblock(); ++b) {
      off[b] = tot;
      tot += 2LL * tt->g.blocks[b].s;
    }
    double *norms = nullptr;
    HB_CUDA(cudaMalloc((void **)&norms, sizeof(double) * std::max(tot, 1LL)));
    std::vector<NormDesc> nd;
    std::vector<BalanceDesc> bd;
    for (int b = 0; b < gt.nblock(); ++b) {
      const BlockDesc &B = tt->g.blocks[b];
      if (B.s == 0) continue;
      double *U = tt->arena + B.u_off, *V = tt->arena + B.v_off;
      nd.push_back(NormDesc{U, B.m, B.m, B.s, norms + off[b]});
      nd.push_back(NormDesc{V, B.n, B.n, B.s, norms + off[b] + B.s});
      bd.push_back(BalanceDesc{U, V, B.m, B.n, B.s, norms + off[b], norms + off[b] + B.s});
    }
    column_norms2(nd, s);
    BalanceDesc *dbd = upload(bd, s);
    for (size_t o = 0; o < bd.size(); o += 65535) {
      balance_kernel<<<dim3(64, (unsigned)std::min<size_t>(65535, bd.size() - o)), 128, 0, s>>>(
          dbd + o);
      HB_LAUNCHED();
    }
    HB_CUDA(cudaStreamSynchronize(s));
    cudaFree(d);
    cudaFree(dbd);
    cudaFree(norms);
  }
  t.transposed = tt;
  return *tt;
}

}  // namespace

void product_mixed_op(DeviceTree &t, ProdOp op, const double *X, int k, long long ldx, double *Y,
                      long long ldy, cudaStream_t s, int min_depth) {
  if (op == ProdOp::N) {
    product_mixed(t, X, k, ldx, Y, ldy, s, min_depth);
    return;
  }
  if (k <= 0 || t.g.n == 0) return;
  DeviceTree *tt;
  {
    std::lock_guard<std::mutex> lk(t.plan_mutex);
    tt = &transposed_tree(t, s);
  }
  if (op == ProdOp::T) {
    product_mixed(*tt, X, k, ldx, Y, ldy, s, min_depth);
    return;
  }
  // X H with X k x n (ld ldx): (X H)^T = H^T X^T
  const int n = t.g.n;
  HB_REQUIRE(ldx >= k && ldy >= k, INPUT_ERROR, "leading dimension below k");
  double *xt = dev_alloc(2 * (size_t)n * k, s);
  double *yt = xt + (size_t)n * k;
  transpose(X, ldx, k, n, xt, n, s);
  try {
    product_mixed(*tt, xt, k, n, yt, n, s, min_depth);
  } catch (...) {
    dev_free(xt, s);
    throw;
  }
  transpose(yt, n, n, k, Y, ldy, s);
  dev_free(xt, s);
}

// ---- many trees, one launch per step -------------------------------------------------

struct MixedBatch {
  double *base = nullptr;
  CopyRange *pre = nullptr, *mid = nullptr;
  int npre = 0, nmid = 0;
  MaxBatch max_x, max_w;
  SliceBatch sl_xa, sl_xb, sl_wb;
  OzSeg *seg1 = nullptr, *seg2 = nullptr;
  OzTile *tile1 = nullptr, *tile2 = nullptr;
  int ntile1 = 0, ntile2 = 0;
  int *start1 = nullptr, *start2 = nullptr;   // per-CTA tile runs (ozaki_schedule)
  int grid1 = 0, grid2 = 0;
  int *status = nullptr;
  ~MixedBatch() {
    for (void *p : {(void *)pre, (void *)mid, (void *)max_x.d, (void *)max_w.d, (void *)sl_xa.d,
                    (void *)sl_xb.d, (void *)sl_wb.d, (void *)seg1, (void *)seg2, (void *)tile1,
                    (void *)tile2, (void *)start1, (void *)start2, (void *)status})
      if (p) cudaFree(p);
  }
};

void MixedBatchDeleter::operator()(MixedBatch *b) const { delete b; }

std::unique_ptr<MixedBatch, MixedBatchDeleter> mixed_batch_build(const std::vector<MixedItem> &items,
                                                                 cudaStream_t s) {
  std::unique_ptr<MixedBatch, MixedBatchDeleter> B(new MixedBatch);
  for (size_t i = 0; i < items.size(); ++i)
    for (size_t j = 0; j < i; ++j)
      HB_REQUIRE(items[i].t != items[j].t, INPUT_ERROR,
                 "a mixed-precision batch takes each tree once");
  std::vector<CopyRange> pre, mid;
  std::vector<OzSeg> s1, s2;
  std::vector<OzTile> t1, t2;
  std::vector<long long> work1;
  std::vector<MaxJob> mx, mw;
  std::vector<SliceJob> sx, sxb, sb;
  // outputs are addressed from the lowest output pointer
  const double *base = nullptr;
  std::vector<MixedPlan *> plans;
  for (const MixedItem &it : items) {
    DeviceTree &t = *it.t;
    HB_REQUIRE(it.k > 0 && it.ldx >= t.g.n && it.ldy >= t.g.n, INPUT_ERROR,
               "leading dimension below n");
    std::lock_guard<std::mutex> lk(t.plan_mutex);
    MixedState &st = mixed_state(t, s);
    plans.push_back(&mixed_plan(t, st, it.k, it.ldx, it.ldy, s));
    for (const double *p : {(const double *)plans.back()->w, (const double *)it.Y})
      if (!base || p < base) base = p;
  }
  B->base = const_cast<double *>(base);
  for (size_t i = 0; i < items.size(); ++i) {
    const MixedItem &it = items[i];
    MixedPlan &P = *plans[i];
    pre.push_back(CopyRange{P.xmax, nullptr, it.k});
    if (P.w_zero) pre.push_back(CopyRange{P.w, nullptr, P.w_zero});
    mid.push_back(CopyRange{P.fmax, P.xmax, it.k});
    const long long wrel = P.w - base, yrel = it.Y - base;
    const int o1 = (int)s1.size(), o2 = (int)s2.size();
    s1.insert(s1.end(), P.hs1.begin(), P.hs1.end());
    s2.insert(s2.end(), P.hs2.begin(), P.hs2.end());
    for (OzTile tl : P.ht1) {
      work1.push_back((long long)P.hs1[tl.seg0].nkb * tl.nw);
      tl.seg0 += o1;
      tl.c_off += wrel;
      t1.push_back(tl);
    }
    for (OzTile tl : P.ht2) {
      tl.seg0 += o2;
      tl.c_off += yrel;
      t2.push_back(tl);
    }
    auto with_x = [&](std::vector<SliceJob> v, std::vector<SliceJob> &dst) {
      for (SliceJob j : v) {
        if (!j.src) j.src = it.X;
        dst.push_back(j);
      }
    };
    for (MaxJob j : P.hmx) {
      if (!j.src) j.src = it.X;
      mx.push_back(j);
    }
    mw.insert(mw.end(), P.hmw.begin(), P.hmw.end());
    with_x(P.hsx, sx);
    with_x(P.hsxb, sxb);
    with_x(P.hsb, sb);
  }
  std::vector<int> order(t1.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work1[a] > work1[b]; });
  std::vector<OzTile> t1s;
  for (int i : order) t1s.push_back(t1[i]);
  B->pre = upload(pre, s);
  B->npre = (int)pre.size();
  B->mid = upload(mid, s);
  B->nmid = (int)mid.size();
  B->max_x = ozaki_max_batch(mx, s);
  B->max_w = ozaki_max_batch(mw, s);
  B->sl_xa = ozaki_slice_batch(sx, s);
  B->sl_xb = ozaki_slice_batch(sxb, s);
  B->sl_wb = ozaki_slice_batch(sb, s);
  B->grid1 = ozaki_grid((int)t1s.size());
  B->grid2 = ozaki_grid((int)t2.size());
  B->start1 = upload(ozaki_schedule(t1s, s1, B->grid1), s);
  B->start2 = upload(ozaki_schedule(t2, s2, B->grid2), s);
  B->seg1 = upload(s1, s);
  B->seg2 = upload(s2, s);
  B->tile1 = upload(t1s, s);
  B->tile2 = upload(t2, s);
  B->ntile1 = (int)t1s.size();
  B->ntile2 = (int)t2.size();
  B->status = dalloc<int>(1);
  HB_CUDA(cudaMemsetAsync(B->status, 0, sizeof(int), s));
  HB_CUDA(cudaStreamSynchronize(s));
  return B;
}

void mixed_batch_run(MixedBatch &B, cudaStream_t s) {
  ozaki_ranges(B.pre, B.npre, s);
  ozaki_max(B.max_x, nullptr, s);
  ozaki_slice(B.sl_xa, nullptr, s);
  ozaki_ranges(B.mid, B.nmid, s);
  ozaki_gemm(B.seg1, B.tile1, B.start1, B.grid1, B.base, B.status, s);
  ozaki_max(B.max_w, nullptr, s);
  ozaki_slice(B.sl_xb, nullptr, s);
  ozaki_slice(B.sl_wb, nullptr, s);
  ozaki_gemm(B.seg2, B.tile2, B.start2, B.grid2, B.base, B.status, s);
}

int mixed_batch_status(MixedBatch &B, cudaStream_t s) {
  int v = 0;
  HB_CUDA(cudaMemcpyAsync(&v, B.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  HB_CUDA(cudaMemsetAsync(B.status, 0, sizeof(int), s));
  return v;
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
