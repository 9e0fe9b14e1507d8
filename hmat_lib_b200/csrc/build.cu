// Dense -> HODLR construction (replaces hmat_lib src/constructors.c:629-704:
// copy_diagonal_blocks :212, compress_matrix :449, compress_off_diagonal
// :308).  Off-diagonal blocks of all levels are disjoint, so every block of
// every level is compressed in the same batched launches (the reference
// walks levels bottom-up with one OpenMP task per block).
#include <algorithm>
#include <chrono>

#include "build.h"
#include "jacobi.h"

namespace hb {

std::shared_ptr<DeviceTree> build_from_dense(const Geometry &g_in, const double *d_A,
                                             long long lda, double tol, cudaStream_t stream,
                                             int *svd_status, BuildStats *stats) {
  auto t0 = std::chrono::steady_clock::now();
  Geometry g = g_in;
  const int nb = g.nblock();
  *svd_status = SUCCESS;

  // ---- exact path: one Jacobi SVD per block --------------------------------
  std::vector<JacobiProb> probs;
  std::vector<int> prob_block;
  long long scratch = 0;
  int max_c = 0;
  struct Slots { long long ws, u, v, sig; };
  std::vector<Slots> slots;
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &B = g.blocks[b];
    const int C = std::min(B.m, B.n);
    if (C == 0) continue;
    Slots s;
    s.ws = scratch;
    scratch += jacobi_workspace(B.m, B.n);
    s.u = scratch;
    scratch += align_up((long long)B.m * C);
    s.v = scratch;
    scratch += align_up((long long)B.n * C);
    s.sig = scratch;
    scratch += align_up(C);
    slots.push_back(s);
    prob_block.push_back(b);
    max_c = std::max(max_c, C);
  }
  const int np = (int)prob_block.size();
  double *work = dev_alloc(scratch, stream);
  int *d_rank = nullptr, *d_status = nullptr;
  JacobiProb *d_probs = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d_rank, sizeof(int) * (np + 1), stream));
  d_status = d_rank + np;
  HB_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), stream));
  for (int p = 0; p < np; ++p) {
    const BlockDesc &B = g.blocks[prob_block[p]];
    const int R = std::max(B.m, B.n), C = std::min(B.m, B.n);
    JacobiProb jp;
    jp.A = d_A + B.r0 + (long long)B.c0 * lda;
    jp.lda = lda;
    jp.m = B.m;
    jp.n = B.n;
    jp.G = work + slots[p].ws;
    jp.W = jp.G + align_up((long long)R * C);
    jp.U = work + slots[p].u;
    jp.ldu = B.m;
    jp.V = work + slots[p].v;
    jp.ldv = B.n;
    jp.sigma = work + slots[p].sig;
    jp.rank = d_rank + p;
    probs.push_back(jp);
  }
  if (np) {
    HB_CUDA(cudaMallocAsync((void **)&d_probs, sizeof(JacobiProb) * np, stream));
    HB_CUDA(cudaMemcpyAsync(d_probs, probs.data(), sizeof(JacobiProb) * np,
                            cudaMemcpyHostToDevice, stream));
    JacobiParams prm;
    prm.tol = tol;
    prm.trunc = Truncation::Relative;
    prm.scale_u = 1;
    prm.max_sweeps = (int)option("jacobi_max_sweeps", 60);
    jacobi_svd_batched(d_probs, np, prm, d_status, max_c, stream);
  }
  std::vector<int> ranks(np + 1, 0);
  HB_CUDA(cudaMemcpyAsync(ranks.data(), d_rank, sizeof(int) * (np + 1), cudaMemcpyDeviceToHost,
                          stream));
  HB_CUDA(cudaStreamSynchronize(stream));
  *svd_status = ranks[np];
  for (auto &B : g.blocks) B.s = 0;
  for (int p = 0; p < np; ++p) g.blocks[prob_block[p]].s = ranks[p];

  // ---- arena: leaves copied from the input, factors from the scratch -------
  std::shared_ptr<DeviceTree> dt = dtree_create(g, stream);
  std::vector<CopyDesc> copies;
  for (int i = 0; i < g.nleaf(); ++i) {
    const LeafDesc &L = dt->leaves[i];
    if (L.m == 0) continue;
    copies.push_back(CopyDesc{d_A + L.r0 + (long long)L.r0 * lda, lda, dt->arena + L.off, L.m,
                              L.m, L.m});
  }
  for (int p = 0; p < np; ++p) {
    const BlockDesc &B = dt->g.blocks[prob_block[p]];
    if (B.s == 0) continue;
    copies.push_back(CopyDesc{probs[p].U, B.m, dt->arena + B.u_off, B.m, B.m, B.s});
    copies.push_back(CopyDesc{probs[p].V, B.n, dt->arena + B.v_off, B.n, B.n, B.s});
  }
  if (!copies.empty()) {
    CopyDesc *d_copies = nullptr;
    HB_CUDA(cudaMallocAsync((void **)&d_copies, sizeof(CopyDesc) * copies.size(), stream));
    HB_CUDA(cudaMemcpyAsync(d_copies, copies.data(), sizeof(CopyDesc) * copies.size(),
                            cudaMemcpyHostToDevice, stream));
    copy2d_batched(d_copies, (int)copies.size(), stream);
    dev_free(d_copies, stream);
  }
  dev_free(d_probs, stream);
  dev_free(d_rank, stream);
  dev_free(work, stream);
  HB_CUDA(cudaStreamSynchronize(stream));
  if (stats) {
    stats->exact_blocks = np;
    stats->seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return dt;
}

}  // namespace hb
