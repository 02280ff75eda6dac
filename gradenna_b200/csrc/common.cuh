// Shared host/device helpers for the gradenna_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/gradenna_b200.h"

namespace gdn {

// Thread-local last-error message returned by gdn_last_error().
void set_error(const char* fmt, ...);
const char* last_error();

struct Status {
  int code = GDN_OK;
  bool ok() const { return code == GDN_OK; }
};

#define GDN_TRY_CUDA(expr)                                                   \
  do {                                                                       \
    cudaError_t e_ = (expr);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      ::gdn::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                  \
      return e_ == cudaErrorMemoryAllocation ? GDN_ERR_OOM : GDN_ERR_CUDA;   \
    }                                                                        \
  } while (0)

#define GDN_BAD_ARG(...)            \
  do {                              \
    ::gdn::set_error(__VA_ARGS__);  \
    return GDN_ERR_BAD_ARG;         \
  } while (0)

// Bump allocator over one workspace block: every sub-buffer is 256-byte
// aligned so vector loads and TMA descriptors can use it.
struct Carve {
  size_t off = 0;
  template <typename X>
  size_t take(size_t count) {
    off = (off + 255) & ~size_t(255);
    size_t at = off;
    off += count * sizeof(X);
    return at;
  }
  size_t bytes() const { return (off + 255) & ~size_t(255); }
};

// Count of kernels this library launched (see gdn_kernel_launches).
void count_launches(uint64_t n);
uint64_t total_launches();

// Device time of one run's time loop for gdn_tm_loop_stats: CUDA events
// recorded on the caller's stream before and after the loop, resolved
// lazily by the stats call. `blocks` counts launches of the dominant kernel
// over the whole grid (TB-step blocks in 2D, time steps in 3D).
class LoopTimer {
 public:
  LoopTimer(cudaStream_t s, double cell_steps, int64_t blocks);
  void stop(bool ok);
  ~LoopTimer();

 private:
  void release();
  cudaEvent_t a_ = nullptr, b_ = nullptr;
  cudaStream_t s_;
  double cells_;
  int64_t blocks_;
};

// A private non-blocking stream per device used only to capture graphs; the
// captured graphs are launched on the caller's stream.
cudaStream_t capture_stream();
// A second private stream per device for parallel branches inside captures.
cudaStream_t capture_side_stream();

template <typename T>
struct Cplx;
template <>
struct Cplx<float> {
  using type = float2;
};
template <>
struct Cplx<double> {
  using type = double2;
};

inline __host__ __device__ long long div_up(long long a, long long b) { return (a + b - 1) / b; }

}  // namespace gdn
