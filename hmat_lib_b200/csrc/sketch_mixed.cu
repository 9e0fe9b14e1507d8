// The build's sketch products on the int8 tensor cores (see sketch_mixed.h).
#include <algorithm>

#include "dtree.h"
#include "sketch_mixed.h"

namespace hb {

namespace {

long long cdiv(long long a, long long b) { return (a + b - 1) / b; }
int pad16(int x) { return (x + 15) / 16 * 16; }

template <class T>
T *upload(const std::vector<T> &v, cudaStream_t s, std::vector<void *> &keep) {
  T *d = nullptr;
  HB_CUDA(cudaMalloc((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1)));
  keep.push_back(d);
  if (!v.empty())
    h2d_async(d, v.data(), sizeof(T) * v.size(), s);
  return d;
}

}  // namespace

SketchMixed::SketchMixed(const std::vector<SketchMixedBlock> &blocks, cudaStream_t s)
    : blocks_(blocks), stream_(s) {
  const int nb = (int)blocks.size();
  row_off_.resize(nb);
  col_off_.resize(nb);
  rexp_off_.resize(nb);
  cexp_off_.resize(nb);
  long long bytes = 0, nexp = 0;
  for (int i = 0; i < nb; ++i) {
    const SketchMixedBlock &B = blocks[i];
    HB_REQUIRE(B.m % kOzKBlock == 0 && B.n % kOzKBlock == 0, INPUT_ERROR,
               "int8 sketches need block sizes that are multiples of 32");
    HB_REQUIRE(B.m <= kOzMaxK && B.n <= kOzMaxK, INPUT_ERROR,
               "int8 sketches: block longer than 65536");
    row_off_[i] = bytes;
    bytes += cdiv(B.m, kOzRowsA) * (B.n / kOzKBlock) * (long long)kOzABlock;
    col_off_[i] = bytes;
    bytes += cdiv(B.n, kOzRowsA) * (B.m / kOzKBlock) * (long long)kOzABlock;
    rexp_off_[i] = nexp;
    nexp += B.m;
    cexp_off_[i] = nexp;
    nexp += B.n;
  }
  // stream-ordered (the device's pool, kept mapped): a synchronous cudaMalloc
  // of the slices (gigabytes) competed with the pool for physical memory
  keep_pool_memory();
  HB_CUDA(cudaMallocAsync((void **)&slices_, std::max<long long>(bytes, 1), s));
  HB_CUDA(cudaMallocAsync((void **)&exps_, sizeof(int) * std::max<long long>(nexp, 1), s));
  HB_CUDA(cudaMallocAsync((void **)&status_, sizeof(int), s));
  HB_CUDA(cudaMemsetAsync(status_, 0, sizeof(int), s));
  unsigned long long *maxabs = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&maxabs, sizeof(unsigned long long) * std::max(nexp, 1LL), s));
  HB_CUDA(cudaMemsetAsync(maxabs, 0, sizeof(unsigned long long) * std::max(nexp, 1LL), s));
  std::vector<MaxJob> mj;
  std::vector<SliceJob> rows, cols;
  for (int i = 0; i < nb; ++i) {
    const SketchMixedBlock &B = blocks[i];
    // rows of A_b (for A Omega): lines adjacent in memory, K = columns
    mj.push_back(MaxJob{B.A, 1, B.lda, B.m, B.n, maxabs + rexp_off_[i], 0});
    rows.push_back(SliceJob{B.A, 1, B.lda, B.m, B.n, kOzRowsA, (int)cdiv(B.m, kOzRowsA), 0,
                            B.n / kOzKBlock, slices_ + row_off_[i],
                            (long long)(B.n / kOzKBlock) * kOzABlock, maxabs + rexp_off_[i],
                            exps_ + rexp_off_[i], 0});
    // columns of A_b (for A^T Q): K contiguous
    mj.push_back(MaxJob{B.A, B.lda, 1, B.n, B.m, maxabs + cexp_off_[i], 0});
    cols.push_back(SliceJob{B.A, B.lda, 1, B.n, B.m, kOzRowsA, (int)cdiv(B.n, kOzRowsA), 0,
                            B.m / kOzKBlock, slices_ + col_off_[i],
                            (long long)(B.m / kOzKBlock) * kOzABlock, maxabs + cexp_off_[i],
                            exps_ + cexp_off_[i], 0});
  }
  MaxBatch bm = ozaki_max_batch(mj, s);
  SliceBatch br = ozaki_slice_batch(rows, s), bc = ozaki_slice_batch(cols, s);
  ozaki_max(bm, nullptr, s);
  ozaki_slice(br, nullptr, s);
  ozaki_slice(bc, nullptr, s);
  HB_CUDA(cudaStreamSynchronize(s));
  for (void *p : {(void *)bm.d, (void *)br.d, (void *)bc.d})
    if (p) cudaFree(p);
  cudaFreeAsync(maxabs, s);
}

SketchMixed::~SketchMixed() {
  for (void *p : {(void *)slices_, (void *)exps_, (void *)status_})
    if (p) cudaFreeAsync(p, stream_);
  cudaStreamSynchronize(stream_);
  for (void *p : keep_)
    if (p) cudaFree(p);
}

void SketchMixed::multiply(bool transA, const std::vector<Call> &calls, cudaStream_t s) {
  if (calls.empty()) return;
  // scratch of every call: column maxima and exponents of X, its slices
  long long sbytes = 0, nw_total = 0;
  std::vector<long long> xs_off(calls.size()), xe_off(calls.size());
  std::vector<int> nws(calls.size()), njbs(calls.size()), Ks(calls.size());
  for (size_t c = 0; c < calls.size(); ++c) {
    const Call &C = calls[c];
    const SketchMixedBlock &B = blocks_[C.block];
    Ks[c] = transA ? B.m : B.n;
    nws[c] = std::min(kOzMaxNw, pad16(C.w));
    njbs[c] = (int)cdiv(C.w, nws[c]);
    xs_off[c] = sbytes;
    sbytes += (long long)njbs[c] * (Ks[c] / kOzKBlock) * oz_bblock(nws[c]);
    xe_off[c] = nw_total;
    nw_total += C.w;
  }
  uint8_t *xsl = nullptr;
  unsigned long long *xmax = nullptr;
  int *xexp = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&xsl, std::max(sbytes, 1LL), s));
  HB_CUDA(cudaMallocAsync((void **)&xmax, sizeof(unsigned long long) * std::max(nw_total, 1LL), s));
  HB_CUDA(cudaMallocAsync((void **)&xexp, sizeof(int) * std::max(nw_total, 1LL), s));
  HB_CUDA(cudaMemsetAsync(xmax, 0, sizeof(unsigned long long) * std::max(nw_total, 1LL), s));
  std::vector<MaxJob> mj;
  std::vector<SliceJob> sj;
  const double *cbase = nullptr;
  for (const Call &C : calls)
    if (!cbase || C.Y < cbase) cbase = C.Y;
  std::vector<OzSeg> segs;
  std::vector<OzTile> tiles;
  for (size_t c = 0; c < calls.size(); ++c) {
    const Call &C = calls[c];
    const SketchMixedBlock &B = blocks_[C.block];
    const int K = Ks[c], nkb = K / kOzKBlock, nw = nws[c];
    const int rowsA = transA ? B.n : B.m;
    // X: K x w column-major -> columns are the lines, K contiguous
    mj.push_back(MaxJob{C.X, C.ldx, 1, C.w, K, xmax + xe_off[c], 0});
    sj.push_back(SliceJob{C.X, C.ldx, 1, C.w, K, nw, njbs[c], 0, nkb, xsl + xs_off[c],
                          (long long)nkb * oz_bblock(nw), xmax + xe_off[c], xexp + xe_off[c], 0});
    const uint8_t *aslices = slices_ + (transA ? col_off_[C.block] : row_off_[C.block]);
    const int *aexp = exps_ + (transA ? cexp_off_[C.block] : rexp_off_[C.block]);
    for (int i = 0; i * kOzRowsA < rowsA; ++i)
      for (int j = 0; j < njbs[c]; ++j) {
        OzTile t{};
        t.seg0 = (int)segs.size();
        t.nseg = 1;
        t.rows = std::min(kOzRowsA, rowsA - i * kOzRowsA);
        t.cols = std::min(nw, C.w - j * nw);
        t.nw = nw;
        t.atomic = 0;
        t.c_off = (long long)(C.Y - cbase) + (long long)i * kOzRowsA + (long long)j * nw * C.ldy;
        t.ldc = C.ldy;
        t.rexp = aexp + i * kOzRowsA;
        t.cexp = xexp + xe_off[c] + j * nw;
        t.rmax = nullptr;
        segs.push_back(OzSeg{aslices + (long long)i * nkb * kOzABlock,
                             xsl + xs_off[c] + (long long)j * nkb * oz_bblock(nw), nkb, 0});
        tiles.push_back(t);
      }
  }
  MaxBatch bm = ozaki_max_batch(mj, s);
  SliceBatch bs = ozaki_slice_batch(sj, s);
  keep_.push_back(bm.d);
  keep_.push_back(bs.d);
  const int grid = ozaki_grid((int)tiles.size());
  const std::vector<int> starts = ozaki_schedule(tiles, segs, grid);
  OzSeg *d_segs = upload(segs, s, keep_);
  OzTile *d_tiles = upload(tiles, s, keep_);
  int *d_starts = upload(starts, s, keep_);
  ozaki_max(bm, nullptr, s);
  ozaki_slice(bs, nullptr, s);
  ozaki_gemm(d_segs, d_tiles, d_starts, grid, const_cast<double *>(cbase), status_, s);
  cudaFreeAsync(xsl, s);
  cudaFreeAsync(xmax, s);
  cudaFreeAsync(xexp, s);
}

int SketchMixed::status(cudaStream_t s) {
  int v = 0;
  HB_CUDA(cudaMemcpyAsync(&v, status_, sizeof(int), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  return v ? SVD_FAILURE : SUCCESS;
}

}  // namespace hb
