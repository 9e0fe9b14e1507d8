// On-disk format of a device tree (hodlr_b200_tree_save / _load).  hmat_lib
// has no serialisation; a tree built once (seconds at n = 65536) can be
// reloaded in the time it takes to read the file.
//
// Layout, little-endian 64-bit words and doubles:
//   "HODLRB20" magic, version (1), height h, n,
//   2^h leaf sizes, 2 (2^h - 1) ranks in block order b = 2(2^d - 1 + j) + (c - 1),
//   every leaf (m x m, column-major) in order, then for every block U (m x s)
//   and V (n x s), column-major, no padding,
//   FNV-1a 64-bit hash of every byte before it.
// Loading validates the header (sizes add up, ranks within the block
// dimensions, the file length) before it allocates anything and checks the
// hash before it returns the tree.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/hmat_lib/hodlr_b200.h"
#include "dtree.h"

using namespace hb;

namespace {

constexpr char kMagic[8] = {'H', 'O', 'D', 'L', 'R', 'B', '2', '0'};
constexpr long long kVersion = 1;
constexpr int kMaxHeight = 30;

struct Hash {
  uint64_t h = 1469598103934665603ULL;
  void add(const void *p, size_t n) {
    auto *c = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) {
      h ^= c[i];
      h *= 1099511628211ULL;
    }
  }
};

struct File {
  FILE *f = nullptr;
  File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

struct Writer {
  FILE *f;
  Hash hash;
  void put(const void *p, size_t bytes) {
    HB_REQUIRE(std::fwrite(p, 1, bytes, f) == bytes, INPUT_ERROR, "tree file: write failed");
    hash.add(p, bytes);
  }
  void word(long long v) { put(&v, sizeof v); }
};

struct Reader {
  FILE *f;
  Hash hash;
  void get(void *p, size_t bytes) {
    HB_REQUIRE(std::fread(p, 1, bytes, f) == bytes, INPUT_ERROR,
               "tree file: shorter than its header says");
    hash.add(p, bytes);
  }
  long long word() {
    long long v = 0;
    get(&v, sizeof v);
    return v;
  }
};

// Element offsets of every leaf, then every U and V, in file order.
template <class F>
void for_each_piece(const DeviceTree &t, F fn) {
  const Geometry &g = t.g;
  for (int i = 0; i < g.nleaf(); ++i)
    fn(t.leaves[i].off, (long long)g.leaf_m[i] * g.leaf_m[i]);
  for (const BlockDesc &b : g.blocks) {
    fn(b.u_off, (long long)b.m * b.s);
    fn(b.v_off, (long long)b.n * b.s);
  }
}

}  // namespace

extern "C" {

int hodlr_b200_tree_save(hodlr_b200_tree t, const char *path) {
  if (!t || !path) return INPUT_ERROR;
  try {
    const DeviceTree &dt = *t->p;
    const Geometry &g = dt.g;
    cudaStream_t s = lib_stream();
    std::vector<double> img(dt.arena_elems);
    if (dt.arena_elems)
      HB_CUDA(cudaMemcpyAsync(img.data(), dt.arena, sizeof(double) * dt.arena_elems,
                              cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    File file(path, "wb");
    HB_REQUIRE(file.f != nullptr, INPUT_ERROR, std::string("tree file: cannot create ") + path);
    Writer w{file.f};
    w.put(kMagic, sizeof kMagic);
    w.word(kVersion);
    w.word(g.h);
    w.word(g.n);
    for (int m : g.leaf_m) w.word(m);
    for (const BlockDesc &b : g.blocks) w.word(b.s);
    for_each_piece(dt, [&](long long off, long long count) {
      if (count) w.put(&img[off], sizeof(double) * count);
    });
    const uint64_t digest = w.hash.h;
    HB_REQUIRE(std::fwrite(&digest, 1, sizeof digest, file.f) == sizeof digest, INPUT_ERROR,
               "tree file: write failed");
    return SUCCESS;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.code;
  }
}

int hodlr_b200_tree_load(const char *path, hodlr_b200_tree *out) {
  if (!path || !out) return INPUT_ERROR;
  try {
    File file(path, "rb");
    HB_REQUIRE(file.f != nullptr, INPUT_ERROR, std::string("tree file: cannot open ") + path);
    std::fseek(file.f, 0, SEEK_END);
    const long long length = std::ftell(file.f);
    std::fseek(file.f, 0, SEEK_SET);
    Reader r{file.f};
    char magic[8];
    r.get(magic, sizeof magic);
    HB_REQUIRE(std::memcmp(magic, kMagic, sizeof magic) == 0, INPUT_ERROR,
               "tree file: not a tree file");
    HB_REQUIRE(r.word() == kVersion, INPUT_ERROR, "tree file: unknown version");
    const long long h = r.word(), n = r.word();
    HB_REQUIRE(h >= 1 && h <= kMaxHeight && n >= 0 && n <= (1LL << 31) - 1, INPUT_ERROR,
               "tree file: bad height or size");
    std::vector<int> leaf(1LL << h);
    long long sum = 0;
    for (auto &m : leaf) {
      const long long v = r.word();
      HB_REQUIRE(v >= 0 && v <= n, INPUT_ERROR, "tree file: bad leaf size");
      m = (int)v;
      sum += v;
    }
    HB_REQUIRE(sum == n, INPUT_ERROR, "tree file: leaf sizes do not add up to n");
    Geometry g = geometry_from_leaves((int)h, leaf);
    long long data = 0;
    for (int m : leaf) data += (long long)m * m;
    for (BlockDesc &b : g.blocks) {
      const long long v = r.word();
      HB_REQUIRE(v >= 0 && v <= std::min(b.m, b.n), INPUT_ERROR, "tree file: bad rank");
      b.s = (int)v;
      data += v * (b.m + b.n);
    }
    const long long expect = (long long)sizeof kMagic + 8LL * (3 + leaf.size() + g.blocks.size()) +
                             8LL * data + (long long)sizeof(uint64_t);
    HB_REQUIRE(length == expect, INPUT_ERROR, "tree file: length does not match its header");
    cudaStream_t s = lib_stream();
    std::shared_ptr<DeviceTree> dt = dtree_create(g, s);
    std::vector<double> img(dt->arena_elems, 0.0);
    for_each_piece(*dt, [&](long long off, long long count) {
      if (count) r.get(&img[off], sizeof(double) * count);
    });
    uint64_t digest = 0;
    HB_REQUIRE(std::fread(&digest, 1, sizeof digest, file.f) == sizeof digest &&
                   digest == r.hash.h,
               INPUT_ERROR, "tree file: checksum mismatch (corrupt file)");
    if (dt->arena_elems)
      HB_CUDA(cudaMemcpyAsync(dt->arena, img.data(), sizeof(double) * dt->arena_elems,
                              cudaMemcpyHostToDevice, s));
    HB_CUDA(cudaStreamSynchronize(s));
    *out = new hodlr_b200_tree_s{dt};
    return SUCCESS;
  } catch (const Error &e) {
    set_last_error(e.msg);
    return e.code;
  }
}

}  // extern "C"
