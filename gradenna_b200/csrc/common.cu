// Error reporting, version string and the per-device capture stream.
#include <atomic>
#include <mutex>

#include "common.cuh"

namespace gdn {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

const char* last_error() { return g_last_error.c_str(); }

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t total_launches() { return g_launches.load(std::memory_order_relaxed); }

cudaStream_t capture_stream() {
  static std::mutex mu;
  static cudaStream_t streams[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64) return nullptr;
  if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
  return streams[dev];
}

cudaStream_t capture_side_stream() {
  static std::mutex mu;
  static cudaStream_t streams[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64) return nullptr;
  if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
  return streams[dev];
}

}  // namespace gdn

extern "C" const char* gdn_version(void) { return "gradenna_b200 0.1 (sm_100a)"; }

extern "C" const char* gdn_last_error(void) { return gdn::last_error(); }

extern "C" uint64_t gdn_kernel_launches(void) { return gdn::total_launches(); }
