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

// Tile binning of point lists (sources, ports, probes, ...): a CSR over the
// tiles of a kernel's grid so each CTA finds the points it owns with two
// loads. `cells` holds (point index, linear cell index) pairs.
struct PointBins {
  std::vector<int> off;    // n_tiles + 1
  std::vector<int2> pts;   // sorted by tile, stable in point order
};

inline PointBins bin_points(int n, const int32_t* pi, const int32_t* pj,
                            int tile_i, int tile_j, int tiles_j, int n_tiles,
                            long long ld) {
  PointBins b;
  b.off.assign(n_tiles + 1, 0);
  b.pts.resize(n);
  std::vector<int> tile_of(n);
  for (int m = 0; m < n; ++m) {
    int t = (pi[m] / tile_i) * tiles_j + (pj[m] / tile_j);
    tile_of[m] = t;
    b.off[t + 1]++;
  }
  for (int t = 0; t < n_tiles; ++t) b.off[t + 1] += b.off[t];
  std::vector<int> cur(b.off.begin(), b.off.end() - 1);
  for (int m = 0; m < n; ++m) {
    int2 v;
    v.x = m;
    v.y = int(pi[m] * ld + pj[m]);
    b.pts[cur[tile_of[m]]++] = v;
  }
  return b;
}

// A private non-blocking stream per device used only to capture graphs; the
// captured graphs are launched on the caller's stream.
cudaStream_t capture_stream();

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
