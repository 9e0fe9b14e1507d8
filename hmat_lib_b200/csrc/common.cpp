// Library-wide state: last error message, launch counter, runtime options.
#include <atomic>
#include <map>
#include <mutex>

#include "common.h"

namespace hb {

namespace {
thread_local std::string g_last_error;
thread_local const char *g_static_error = nullptr;
std::atomic<long long> g_launches{0};
std::mutex g_opt_mutex;
std::map<std::string, double> &opts() {
  static std::map<std::string, double> m;
  return m;
}
}  // namespace

void set_last_error(const std::string &msg) {
  g_static_error = nullptr;
  g_last_error = msg;
}
void set_last_error_static(const char *msg) { g_static_error = msg; }
const char *last_error() { return g_static_error ? g_static_error : g_last_error.c_str(); }

void count_launch(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches() { return g_launches.load(); }

int num_sms() {
  static int cached = 0;
  if (cached == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached = v;
  }
  return cached;
}

double option(const char *name, double dflt) {
  std::lock_guard<std::mutex> lk(g_opt_mutex);
  auto it = opts().find(name);
  return it == opts().end() ? dflt : it->second;
}

void set_option(const std::string &name, double value) {
  std::lock_guard<std::mutex> lk(g_opt_mutex);
  opts()[name] = value;
}

}  // namespace hb
