// Device tree arena, upload / download and the host-tree registry.
#include <atomic>
#include <deque>
#include <vector>
#include <cstring>
#include <unordered_map>

#include "dtree.h"
#include "products.h"

namespace hb {

namespace {
std::mutex g_reg_mutex;
std::unordered_map<const TreeHODLR *, std::shared_ptr<DeviceTree>> g_registry;
}  // namespace

DeviceTree::~DeviceTree() {
  graphs.clear();
  plans.clear();
  mixed.reset();
  transposed.reset();
  if (arena) cudaFree(arena);
  if (d_leaves) cudaFree(d_leaves);
  if (d_blocks) cudaFree(d_blocks);
  if (mv_woff) cudaFree(mv_woff);
  if (mv_w) cudaFree(mv_w);
}

long long DeviceTree::storage() const {
  long long w = 0;
  for (int m : g.leaf_m) w += (long long)m * m;
  for (auto &b : g.blocks) w += (long long)b.s * (b.m + b.n);
  return w;
}

cudaStream_t lib_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  keep_pool_memory();
  cudaStream_t s;
  HB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  streams[dev] = s;
  return s;
}

// Freed stream-ordered memory stays mapped in the device's default pool
// (release threshold unlimited), so that a build, whose sketch rounds
// synchronise with the host, does not unmap its scratch at every
// synchronisation and map it again in the next round.  Option pool_keep = 0,
// set before the library's first allocation on a device, leaves the pool as
// the process configured it.  Applied once per device.
void keep_pool_memory() {
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    (void)cudaGetLastError();
    return;
  }
  const unsigned long long bit = 1ULL << dev;
  if (done.load(std::memory_order_acquire) & bit) return;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (done.load() & bit) return;
  done.fetch_or(bit);
  if (option("pool_keep", 1.0) == 0.0) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  uint64_t keep = ~0ULL;
  if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
    (void)cudaGetLastError();
}

double *dev_alloc(size_t elems, cudaStream_t stream) {
  keep_pool_memory();
  void *p = nullptr;
  HB_CUDA(cudaMallocAsync(&p, std::max<size_t>(elems, 1) * sizeof(double), stream));
  return (double *)p;
}

void dev_free(void *p, cudaStream_t stream) {
  if (p) cudaFreeAsync(p, stream);
}

namespace {

struct PinnedRing {
  char *base = nullptr;
  size_t cap = 0, head = 0;
  bool tried = false;
  struct Span {
    size_t lo, hi;
    cudaEvent_t ev;
  };
  std::deque<Span> live;
  std::vector<cudaEvent_t> spare;
  ~PinnedRing() {
    for (Span &sp : live) cudaEventSynchronize(sp.ev);
    for (Span &sp : live) cudaEventDestroy(sp.ev);
    for (cudaEvent_t e : spare) cudaEventDestroy(e);
    if (base) cudaFreeHost(base);
    (void)cudaGetLastError();
  }
};

constexpr size_t kRingBytes = size_t(64) << 20;

}  // namespace

void h2d_async(void *dst, const void *src, size_t bytes, cudaStream_t stream) {
  if (bytes == 0) return;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  HB_CUDA(cudaStreamIsCapturing(stream, &cap));
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  thread_local std::unordered_map<int, PinnedRing> rings;
  PinnedRing &R = rings[dev];
  if (!R.tried) {
    R.tried = true;
    if (cudaMallocHost((void **)&R.base, kRingBytes) == cudaSuccess) {
      R.cap = kRingBytes;
    } else {
      (void)cudaGetLastError();
      R.base = nullptr;
    }
  }
  const size_t need = (bytes + 255) / 256 * 256;
  if (cap != cudaStreamCaptureStatusNone || !R.base || need > R.cap / 2) {
    HB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
    return;
  }
  // retire finished copies, oldest first
  while (!R.live.empty() && cudaEventQuery(R.live.front().ev) == cudaSuccess) {
    R.spare.push_back(R.live.front().ev);
    R.live.pop_front();
  }
  (void)cudaGetLastError();   // cudaErrorNotReady from the last query
  size_t lo = R.head;
  if (lo + need > R.cap) lo = 0;
  const size_t hi = lo + need;
  // wait for every copy still reading the slot
  for (auto it = R.live.begin(); it != R.live.end();) {
    if (it->lo < hi && lo < it->hi) {
      HB_CUDA(cudaEventSynchronize(it->ev));
      R.spare.push_back(it->ev);
      it = R.live.erase(it);
    } else {
      ++it;
    }
  }
  std::memcpy(R.base + lo, src, bytes);
  HB_CUDA(cudaMemcpyAsync(dst, R.base + lo, bytes, cudaMemcpyHostToDevice, stream));
  cudaEvent_t ev;
  if (!R.spare.empty()) {
    ev = R.spare.back();
    R.spare.pop_back();
  } else {
    HB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  HB_CUDA(cudaEventRecord(ev, stream));
  R.live.push_back(PinnedRing::Span{lo, hi, ev});
  R.head = hi;
}

std::unique_ptr<DeviceTree> dtree_create(const Geometry &g_in, cudaStream_t stream) {
  auto t = std::make_unique<DeviceTree>();
  HB_CUDA(cudaGetDevice(&t->device));
  t->g = g_in;
  Geometry &g = t->g;
  long long off = 0;
  t->leaves.resize(g.nleaf());
  for (int i = 0; i < g.nleaf(); ++i) {
    t->leaves[i] = LeafDesc{(int)g.leaf_off[i], g.leaf_m[i], off};
    off += align_up((long long)g.leaf_m[i] * g.leaf_m[i]);
  }
  for (auto &b : g.blocks) {
    b.u_off = off;
    off += align_up((long long)b.m * b.s);
    b.v_off = off;
    off += align_up((long long)b.n * b.s);
  }
  t->arena_elems = off;
  // from the device's stream-ordered pool (kept mapped, see keep_pool_memory):
  // a build allocates its tree while the GPU waits, and a synchronous
  // cudaMalloc of the arena had to map fresh pages there.  cudaFree releases
  // these allocations like any other.
  keep_pool_memory();
  HB_CUDA(cudaMallocAsync((void **)&t->arena, std::max<long long>(off, 1) * sizeof(double),
                          stream));
  HB_CUDA(cudaMallocAsync((void **)&t->d_leaves,
                          std::max<size_t>(t->leaves.size(), 1) * sizeof(LeafDesc), stream));
  HB_CUDA(cudaMallocAsync((void **)&t->d_blocks,
                          std::max<size_t>(g.blocks.size(), 1) * sizeof(BlockDesc), stream));
  HB_CUDA(cudaMemcpyAsync(t->d_leaves, t->leaves.data(), t->leaves.size() * sizeof(LeafDesc),
                          cudaMemcpyHostToDevice, stream));
  if (!g.blocks.empty())
    HB_CUDA(cudaMemcpyAsync(t->d_blocks, g.blocks.data(), g.blocks.size() * sizeof(BlockDesc),
                            cudaMemcpyHostToDevice, stream));
  // the allocations (stream-ordered on `stream`) and descriptors are ready
  // for use on any stream once this returns
  HB_CUDA(cudaStreamSynchronize(stream));
  return t;
}

void dtree_upload(DeviceTree &t, HODLRInternalNode *root, cudaStream_t stream) {
  const Geometry &g = t.g;
  // gather into one host staging image of the arena, one copy
  std::vector<double> img(t.arena_elems, 0.0);
  for (int i = 0; i < g.nleaf(); ++i) {
    HODLRLeafNode *leaf = diag_leaf(root, g.h, i);
    const long long mm = (long long)g.leaf_m[i] * g.leaf_m[i];
    HB_REQUIRE(mm == 0 || leaf->data.diagonal.data != nullptr, INPUT_ERROR,
               "diagonal leaf without data");
    if (mm) std::memcpy(&img[t.leaves[i].off], leaf->data.diagonal.data, mm * sizeof(double));
  }
  for (int d = 0; d < g.h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      HODLRInternalNode *node = node_at(root, d, j);
      for (int c = 1; c <= 2; ++c) {
        const NodeOffDiagonal &od = node->children[c].leaf->data.off_diagonal;
        const BlockDesc &b = g.blocks[block_index(d, j, c)];
        const long long mu = (long long)b.m * b.s, mv = (long long)b.n * b.s;
        HB_REQUIRE((mu == 0 || od.u != nullptr) && (mv == 0 || od.v != nullptr), INPUT_ERROR,
                   "off-diagonal leaf without factors");
        if (mu) std::memcpy(&img[b.u_off], od.u, mu * sizeof(double));
        if (mv) std::memcpy(&img[b.v_off], od.v, mv * sizeof(double));
      }
    }
  if (t.arena_elems)
    HB_CUDA(cudaMemcpyAsync(t.arena, img.data(), t.arena_elems * sizeof(double),
                            cudaMemcpyHostToDevice, stream));
  HB_CUDA(cudaStreamSynchronize(stream));
}

void dtree_download(const DeviceTree &t, TreeHODLR *host, cudaStream_t stream) {
  const Geometry &g = t.g;
  std::vector<double> img(t.arena_elems);
  if (t.arena_elems)
    HB_CUDA(cudaMemcpyAsync(img.data(), t.arena, t.arena_elems * sizeof(double),
                            cudaMemcpyDeviceToHost, stream));
  HB_CUDA(cudaStreamSynchronize(stream));
  auto copy_out = [&](long long off, long long count) -> double * {
    auto *p = (double *)host_malloc(std::max<long long>(count, 1) * sizeof(double));
    HB_REQUIRE(p != nullptr, ALLOCATION_FAILURE, "host allocation of tree data failed");
    if (count) std::memcpy(p, &img[off], count * sizeof(double));
    return p;
  };
  for (int i = 0; i < g.nleaf(); ++i) {
    HODLRLeafNode *leaf = diag_leaf(host->root, g.h, i);
    leaf->data.diagonal.m = g.leaf_m[i];
    leaf->data.diagonal.data = copy_out(t.leaves[i].off, (long long)g.leaf_m[i] * g.leaf_m[i]);
  }
  for (int d = 0; d < g.h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      HODLRInternalNode *node = node_at(host->root, d, j);
      const int span = 1 << (g.h - d);
      node->m = (int)(g.leaf_off[(j + 1) * span] - g.leaf_off[j * span]);
      for (int c = 1; c <= 2; ++c) {
        NodeOffDiagonal &od = node->children[c].leaf->data.off_diagonal;
        const BlockDesc &b = g.blocks[block_index(d, j, c)];
        od.m = b.m;
        od.n = b.n;
        od.s = b.s;
        od.u = copy_out(b.u_off, (long long)b.m * b.s);
        od.v = copy_out(b.v_off, (long long)b.n * b.s);
      }
    }
}

// FNV-1a over the tree's structure, data pointers and a few values of every
// buffer.  Detects a different tree at a reused address; in-place edits of
// factor values that leave the sampled entries unchanged must be announced
// with hodlr_b200_sync_tree().
uint64_t host_fingerprint(const TreeHODLR *t) {
  uint64_t h = 1469598103934665603ULL;
  auto mix = [&](const void *p, size_t n) {
    auto *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) {
      h ^= c[i];
      h *= 1099511628211ULL;
    }
  };
  auto sample = [&](const double *x, long long count) {
    mix(&x, sizeof(x));
    mix(&count, sizeof(count));
    if (!x || count <= 0) return;
    const long long idx[5] = {0, count / 4, count / 2, (3 * count) / 4, count - 1};
    for (long long i : idx) mix(&x[i], sizeof(double));
  };
  mix(&t->height, sizeof(int));
  const Geometry g = geometry_of(t);
  for (int i = 0; i < g.nleaf(); ++i) {
    HODLRLeafNode *leaf = diag_leaf(t->root, g.h, i);
    sample(leaf->data.diagonal.data, (long long)g.leaf_m[i] * g.leaf_m[i]);
  }
  for (int d = 0; d < g.h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      HODLRInternalNode *node = node_at(t->root, d, j);
      for (int c = 1; c <= 2; ++c) {
        const NodeOffDiagonal &od = node->children[c].leaf->data.off_diagonal;
        mix(&od.s, sizeof(int));
        sample(od.u, (long long)od.m * od.s);
        sample(od.v, (long long)od.n * od.s);
      }
    }
  return h;
}

void register_device_tree(const TreeHODLR *t, std::shared_ptr<DeviceTree> dt) {
  dt->fingerprint = host_fingerprint(t);
  std::lock_guard<std::mutex> lk(g_reg_mutex);
  g_registry[t] = std::move(dt);
}

std::shared_ptr<DeviceTree> device_tree_for(const TreeHODLR *t, cudaStream_t stream) {
  HB_REQUIRE(t != nullptr && t->root != nullptr, INPUT_ERROR, "NULL tree");
  int dev = 0;
  HB_CUDA(cudaGetDevice(&dev));
  const uint64_t fp = host_fingerprint(t);
  {
    std::lock_guard<std::mutex> lk(g_reg_mutex);
    auto it = g_registry.find(t);
    if (it != g_registry.end() && it->second->fingerprint == fp && it->second->device == dev)
      return it->second;
  }
  Geometry g = geometry_of(t);
  std::shared_ptr<DeviceTree> dt = dtree_create(g, stream);
  dtree_upload(*dt, t->root, stream);
  dt->fingerprint = fp;
  std::lock_guard<std::mutex> lk(g_reg_mutex);
  g_registry[t] = dt;
  return dt;
}

void forget_device_tree(const TreeHODLR *t) {
  std::lock_guard<std::mutex> lk(g_reg_mutex);
  g_registry.erase(t);
}

}  // namespace hb
