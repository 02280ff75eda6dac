// 2D TM FDTD time loop for B200 (sm_100a).
//
// Replaces the reference's fused CPU loop gradenna_tm_run_f32/_f64
// (rust/src/lib.rs:89-641) and the JAX scan body of simulate_tm
// (src/gradenna/fdtd2d.py:412-464) with the same per-step semantics:
//
//   H sweep with slab-stored CPML psi (fdtd2d.py:416-428, cpml.py:120-158)
//   -> Mx/My injection -> port Ampere current + Ez^n snapshot (:430-436)
//   -> E sweep with psi (:438-443) -> Jz injection (:444) -> RVS port
//   injection and V record (:446-451) -> running DFT (:453-458) -> probes.
//
// B200 design:
//   * Field state lives in a RING of R slots (ez, hx, hy per slot, rows padded
//     to `ld`). Step n reads slot n%R and writes slot (n+1)%R, so every slot
//     is a snapshot of the fields after one step. The H and E kernels of a
//     step therefore never update in place, and the running DFT is folded
//     into the accumulators once per T = R-1 steps by one kernel that reads
//     T snapshots: accumulator read-modify-write traffic drops by T.
//   * Point work (sources, ports, probes, magnetic currents) is binned by
//     tile on the host; the CTA owning a tile applies it after its sweep, so
//     no extra launches are needed per step.
//   * One chunk of T steps (2T sweeps + DFT fold + step-counter advance) is
//     captured once as a CUDA graph and replayed; kernels read the absolute
//     step index from a device counter.
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace gdn {
namespace tm2d {

constexpr int TJ = 32;  // tile width (contiguous axis)
constexpr int TI = 8;   // tile height
constexpr int KMAX = 16;

template <typename T>
struct Dev {
  int nx, ny, ld, npml, R, n_steps, n_freq, tiles_x;
  long long slot;  // elements per ring slot (3 * nx * ld)
  T* ring;
  const T *ca, *cb, *eps;
  const T *ikx_e, *iky_e, *ikx_h, *iky_h;
  const T *b_ezx_lo, *c_ezx_lo, *b_ezx_hi, *c_ezx_hi;
  const T *b_ezy_lo, *c_ezy_lo, *b_ezy_hi, *c_ezy_hi;
  const T *b_hyx_lo, *c_hyx_lo, *b_hyx_hi, *c_hyx_hi;
  const T *b_hxy_lo, *c_hxy_lo, *b_hxy_hi, *c_hxy_hi;
  T *ezx_lo, *ezx_hi, *ezy_lo, *ezy_hi, *hyx_lo, *hyx_hi, *hxy_lo, *hxy_hi;
  T dt_mu, inv_dx, inv_dy, dx, dy, dz;
  int n_src, n_ports, n_mx, n_my, n_probes;
  const int *src_off, *port_off, *mx_off, *my_off, *probe_off;
  const int2 *src_pts, *port_pts, *mx_pts, *my_pts, *probe_pts;
  const T *cb_src, *src_cur, *cb_vs, *port_vs, *mx_cur, *my_cur;
  int cw;
  const double* cw_env;
  const double2 *src_w, *mx_w, *my_w, *ph_e, *ph_h;
  T *out_probe, *out_v, *out_i;
  const int* step_base;
};

template <typename A>
struct DftDev {
  int lo[3][2], hi[3][2];
  typename Cplx<A>::type* acc[3];
};

// Value of a point source waveform at step n: tabulated, or synthesised from
// CW phasor weights, J(n) = env[n] Re(sum_k W_k conj(ph[n,k])).
template <typename T>
__device__ __forceinline__ T point_value(const Dev<T>& d, const T* cur, const double2* w,
                                         const double2* ph, int n_pts, int m, int n) {
  if (!d.cw) return cur[(long long)n * n_pts + m];
  double s = 0.0;
  for (int k = 0; k < d.n_freq; ++k) {
    double2 a = w[(long long)m * d.n_freq + k];
    double2 p = ph[(long long)n * d.n_freq + k];
    s += a.x * p.x + a.y * p.y;
  }
  return T(d.cw_env[n] * s);
}

template <typename T>
__device__ __forceinline__ void atomic_add(T* p, T v) {
  atomicAdd(p, v);
}

// ---------------------------------------------------------------------------
// H sweep: E^n -> H^{n+1/2}  (fdtd2d.py:416-428; lib.rs:298-375)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TI * TJ) tm_h_sweep(Dev<T> d, int sub) {
  const int n = *d.step_base + sub;
  const int nx = d.nx, ny = d.ny, ld = d.ld, npml = d.npml;
  const T* ez0 = d.ring + (long long)(n % d.R) * d.slot;
  const T* hx0 = ez0 + (long long)nx * ld;
  const T* hy0 = hx0 + (long long)nx * ld;
  T* hx1 = d.ring + (long long)((n + 1) % d.R) * d.slot + (long long)nx * ld;
  T* hy1 = hx1 + (long long)nx * ld;

  const int j = blockIdx.x * TJ + threadIdx.x;
  const int i = blockIdx.y * TI + threadIdx.y;
  const long long c = (long long)i * ld + j;
  if (i < nx && j < ny - 1) {
    const T diff = (ez0[c + 1] - ez0[c]) * d.inv_dy;
    T term = diff;
    if (j < npml) {
      T* ps = d.hxy_lo + (long long)i * npml + j;
      const T p = d.b_hxy_lo[j] * *ps + d.c_hxy_lo[j] * diff;
      *ps = p;
      term = diff * d.iky_h[j] + p;
    } else if (j >= ny - 1 - npml) {
      const int s = j - (ny - 1 - npml);
      T* ps = d.hxy_hi + (long long)i * npml + s;
      const T p = d.b_hxy_hi[s] * *ps + d.c_hxy_hi[s] * diff;
      *ps = p;
      term = diff * d.iky_h[j] + p;
    }
    hx1[c] = hx0[c] - d.dt_mu * term;
  }
  if (i < nx - 1 && j < ny) {
    const T diff = (ez0[c + ld] - ez0[c]) * d.inv_dx;
    T term = diff;
    if (i < npml) {
      T* ps = d.hyx_lo + (long long)i * ny + j;
      const T p = d.b_hyx_lo[i] * *ps + d.c_hyx_lo[i] * diff;
      *ps = p;
      term = diff * d.ikx_h[i] + p;
    } else if (i >= nx - 1 - npml) {
      const int s = i - (nx - 1 - npml);
      T* ps = d.hyx_hi + (long long)s * ny + j;
      const T p = d.b_hyx_hi[s] * *ps + d.c_hyx_hi[s] * diff;
      *ps = p;
      term = diff * d.ikx_h[i] + p;
    }
    hy1[c] = hy0[c] + d.dt_mu * term;
  }

  // Magnetic-current injection on this tile: H -= (dt/mu) M (fdtd2d.py:419-428).
  const int tile = blockIdx.y * gridDim.x + blockIdx.x;
  const int mb = d.mx_off[tile], me = d.mx_off[tile + 1];
  const int yb = d.my_off[tile], ye = d.my_off[tile + 1];
  if (mb < me || yb < ye) {
    __syncthreads();
    const int tid = threadIdx.y * TJ + threadIdx.x;
    for (int q = mb + tid; q < me; q += TI * TJ) {
      const int2 pt = d.mx_pts[q];
      atomic_add(hx1 + pt.y, -(d.dt_mu * point_value(d, d.mx_cur, d.mx_w, d.ph_h, d.n_mx, pt.x, n)));
    }
    for (int q = yb + tid; q < ye; q += TI * TJ) {
      const int2 pt = d.my_pts[q];
      atomic_add(hy1 + pt.y, -(d.dt_mu * point_value(d, d.my_cur, d.my_w, d.ph_h, d.n_my, pt.x, n)));
    }
  }
}

// ---------------------------------------------------------------------------
// E sweep: H^{n+1/2} -> E^{n+1} on the interior, then Jz / ports / probes
// (fdtd2d.py:430-461; lib.rs:389-535)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TI * TJ) tm_e_sweep(Dev<T> d, int sub) {
  const int n = *d.step_base + sub;
  const int nx = d.nx, ny = d.ny, ld = d.ld, npml = d.npml;
  const T* ez0 = d.ring + (long long)(n % d.R) * d.slot;
  T* ez1 = d.ring + (long long)((n + 1) % d.R) * d.slot;
  const T* hx1 = ez1 + (long long)nx * ld;
  const T* hy1 = hx1 + (long long)nx * ld;

  const int j = blockIdx.x * TJ + threadIdx.x;
  const int i = blockIdx.y * TI + threadIdx.y;
  const long long c = (long long)i * ld + j;
  if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
    const T dhy_dx = (hy1[c] - hy1[c - ld]) * d.inv_dx;
    const T dhx_dy = (hx1[c] - hx1[c - 1]) * d.inv_dy;
    T tx = dhy_dx, ty = dhx_dy;
    const int a = i - 1, b = j - 1;
    const int nxi = nx - 2, nyi = ny - 2;
    if (a < npml) {
      T* ps = d.ezx_lo + (long long)a * nyi + b;
      const T p = d.b_ezx_lo[a] * *ps + d.c_ezx_lo[a] * dhy_dx;
      *ps = p;
      tx = dhy_dx * d.ikx_e[a] + p;
    } else if (a >= nxi - npml) {
      const int s = a - (nxi - npml);
      T* ps = d.ezx_hi + (long long)s * nyi + b;
      const T p = d.b_ezx_hi[s] * *ps + d.c_ezx_hi[s] * dhy_dx;
      *ps = p;
      tx = dhy_dx * d.ikx_e[a] + p;
    }
    if (b < npml) {
      T* ps = d.ezy_lo + (long long)a * npml + b;
      const T p = d.b_ezy_lo[b] * *ps + d.c_ezy_lo[b] * dhx_dy;
      *ps = p;
      ty = dhx_dy * d.iky_e[b] + p;
    } else if (b >= nyi - npml) {
      const int s = b - (nyi - npml);
      T* ps = d.ezy_hi + (long long)a * npml + s;
      const T p = d.b_ezy_hi[s] * *ps + d.c_ezy_hi[s] * dhx_dy;
      *ps = p;
      ty = dhx_dy * d.iky_e[b] + p;
    }
    const long long g = (long long)i * ny + j;
    ez1[c] = d.ca[g] * ez0[c] + d.cb[g] * (tx - ty);
  }

  const int tile = blockIdx.y * gridDim.x + blockIdx.x;
  const int sb = d.src_off[tile], se = d.src_off[tile + 1];
  const int pb = d.port_off[tile], pe = d.port_off[tile + 1];
  const int qb = d.probe_off[tile], qe = d.probe_off[tile + 1];
  if (sb < se || pb < pe || qb < qe) {
    const int tid = threadIdx.y * TJ + threadIdx.x;
    __syncthreads();
    // Jz line sources: Ez -= cb_src * J (fdtd2d.py:444).
    for (int q = sb + tid; q < se; q += TI * TJ) {
      const int2 pt = d.src_pts[q];
      atomic_add(ez1 + pt.y, -(d.cb_src[pt.x] * point_value(d, d.src_cur, d.src_w, d.ph_e, d.n_src, pt.x, n)));
    }
    __syncthreads();
    // RVS ports, in port order (fdtd2d.py:430-436, 446-451): all injections
    // on this tile first, then the V/I records.
    if (tid == 0 && pb < pe) {
      for (int q = pb; q < pe; ++q) {
        const int2 pt = d.port_pts[q];
        ez1[pt.y] += -(d.cb_vs[pt.x] * d.port_vs[(long long)n * d.n_ports + pt.x]);
      }
      for (int q = pb; q < pe; ++q) {
        const int2 pt = d.port_pts[q];
        const long long p = pt.y;
        const T cur = (hy1[p] - hy1[p - ld]) * d.dy - (hx1[p] - hx1[p - 1]) * d.dx;
        d.out_i[(long long)n * d.n_ports + pt.x] = cur;
        d.out_v[(long long)n * d.n_ports + pt.x] = T(-0.5) * d.dz * (ez0[p] + ez1[p]);
      }
    }
    __syncthreads();
    for (int q = qb + tid; q < qe; q += TI * TJ) {
      const int2 pt = d.probe_pts[q];
      d.out_probe[(long long)n * d.n_probes + pt.x] = ez1[pt.y];
    }
  }
}

// ---------------------------------------------------------------------------
// Running DFT fold over `cnt` ring snapshots (fdtd2d.py:453-458): for each
// accumulated cell, acc_k += sum_t ph[n0+t, k] * x_t, partial sums in A.
// ---------------------------------------------------------------------------
template <typename T, typename A>
__global__ void __launch_bounds__(256) tm_dft_fold(Dev<T> d, DftDev<A> q, int sub0, int cnt) {
  extern __shared__ unsigned char smem_raw[];
  A* sph = reinterpret_cast<A*>(smem_raw);  // [2 tables][cnt][K][re, im]
  const int n0 = *d.step_base + sub0;
  const int K = d.n_freq;
  for (int idx = threadIdx.x; idx < cnt * K; idx += blockDim.x) {
    const int t = idx / K, k = idx - t * K;
    const double2 pe = d.ph_e[(long long)(n0 + t) * K + k];
    const double2 ph = d.ph_h[(long long)(n0 + t) * K + k];
    sph[2 * idx] = A(pe.x);
    sph[2 * idx + 1] = A(pe.y);
    sph[2 * (cnt * K + idx)] = A(ph.x);
    sph[2 * (cnt * K + idx) + 1] = A(ph.y);
  }
  __syncthreads();
  const int comp = blockIdx.y;
  const int h = q.hi[comp][0] - q.lo[comp][0];
  const int w = q.hi[comp][1] - q.lo[comp][1];
  if (h <= 0 || w <= 0) return;
  const long long count = (long long)h * w;
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= count) return;
  const int ri = int(r / w), rj = int(r - (long long)ri * w);
  const int i = q.lo[comp][0] + ri, j = q.lo[comp][1] + rj;
  const A* ph = sph + (comp == 0 ? 0 : 2 * cnt * K);
  const long long field_off = (long long)comp * d.nx * d.ld + (long long)i * d.ld + j;
  A are[KMAX], aim[KMAX];
#pragma unroll
  for (int k = 0; k < KMAX; ++k) are[k] = aim[k] = A(0);
#pragma unroll 4
  for (int t = 0; t < cnt; ++t) {
    const int slot = (n0 + t + 1) % d.R;
    const A x = A(d.ring[(long long)slot * d.slot + field_off]);
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      if (k < K) {
        are[k] += ph[2 * (t * K + k)] * x;
        aim[k] += ph[2 * (t * K + k) + 1] * x;
      }
    }
  }
  typename Cplx<A>::type* acc = q.acc[comp] + r;
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    if (k < K) {
      typename Cplx<A>::type v = acc[(long long)k * count];
      v.x += are[k];
      v.y += aim[k];
      acc[(long long)k * count] = v;
    }
  }
}

// Total field energy 1/2 (eps Ez^2 + mu0 H^2) dA (fdtd2d.py:160-169), reduced
// in double into eacc[2n] (electric sum) and eacc[2n+1] (magnetic sum).
template <typename T>
__global__ void tm_energy(Dev<T> d, double* eacc, int sub) {
  const int n = *d.step_base + sub;
  const T* ez1 = d.ring + (long long)((n + 1) % d.R) * d.slot;
  const T* hx1 = ez1 + (long long)d.nx * d.ld;
  const T* hy1 = hx1 + (long long)d.nx * d.ld;
  double ue = 0.0, uh = 0.0;
  const long long total = (long long)d.nx * d.ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = int(g / d.ny), j = int(g - (long long)i * d.ny);
    const long long c = (long long)i * d.ld + j;
    const double e = double(ez1[c]);
    ue += double(d.eps[g]) * e * e;
    if (j < d.ny - 1) uh += double(hx1[c]) * double(hx1[c]);
    if (i < d.nx - 1) uh += double(hy1[c]) * double(hy1[c]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    ue += __shfl_down_sync(0xffffffffu, ue, o);
    uh += __shfl_down_sync(0xffffffffu, uh, o);
  }
  __shared__ double sue[32], suh[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sue[wid] = ue;
    suh[wid] = uh;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    ue = lane < nw ? sue[lane] : 0.0;
    uh = lane < nw ? suh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      ue += __shfl_down_sync(0xffffffffu, ue, o);
      uh += __shfl_down_sync(0xffffffffu, uh, o);
    }
    if (lane == 0) {
      atomicAdd(eacc + 2 * n, ue);
      atomicAdd(eacc + 2 * n + 1, uh);
    }
  }
}

template <typename T>
__global__ void tm_energy_finish(const double* eacc, T* out, int n_steps, double cell,
                                     double mu0) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < n_steps) out[n] = T(0.5 * eacc[2 * n] * cell + 0.5 * mu0 * eacc[2 * n + 1] * cell);
}

__global__ void tm_advance(int* step_base, int cnt) { *step_base += cnt; }

// Copy the final ring slot into the caller's unpadded ez/hx/hy.
template <typename T>
__global__ void tm_copy_out(const T* slot, int nx, int ny, int ld, T* ez, T* hx, T* hy) {
  const long long total = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = int(g / ny), j = int(g - (long long)i * ny);
    const long long c = (long long)i * ld + j;
    ez[g] = slot[c];
    if (j < ny - 1) hx[(long long)i * (ny - 1) + j] = slot[(long long)nx * ld + c];
    if (i < nx - 1) hy[g] = slot[2LL * nx * ld + c];
  }
}

template <typename C>
__global__ void tm_dft_scale(C* a, long long count, double s) {
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < count;
       g += (long long)gridDim.x * blockDim.x) {
    C v = a[g];
    v.x *= s;
    v.y *= s;
    a[g] = v;
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

struct Layout {
  int ld = 0, R = 2, T = 32, tiles_x = 0, tiles_y = 0, n_tiles = 0;
  long long slot = 0;
  size_t ring, psi[8], off[5], pts[5], step, eacc, total;
};

static int dft_block_steps(const GdnTmParams* p, size_t slot_bytes) {
  if (p->n_freq <= 0) return 32;
  const size_t budget = size_t(2) << 30;  // ring budget: 2 GiB
  long long t = (long long)(budget / std::max<size_t>(slot_bytes, 1)) - 1;
  t = std::min<long long>(32, std::max<long long>(2, t));
  return int(t);
}

static Layout make_layout(const GdnTmParams* p, size_t esize) {
  Layout L;
  L.ld = int(div_up(p->ny, 32) * 32);
  L.slot = 3LL * p->nx * L.ld;
  L.T = dft_block_steps(p, size_t(L.slot) * esize);
  L.R = p->n_freq > 0 ? L.T + 1 : 2;
  L.tiles_x = L.ld / TJ;
  L.tiles_y = int(div_up(p->nx, TI));
  L.n_tiles = L.tiles_x * L.tiles_y;
  Carve cv;
  L.ring = cv.take<char>(size_t(L.R) * L.slot * esize);
  const int m = p->npml, nx = p->nx, ny = p->ny;
  const size_t psz[8] = {size_t(m) * (ny - 2), size_t(m) * (ny - 2), size_t(nx - 2) * m,
                         size_t(nx - 2) * m,   size_t(m) * ny,       size_t(m) * ny,
                         size_t(nx) * m,       size_t(nx) * m};
  for (int k = 0; k < 8; ++k) L.psi[k] = cv.take<char>(psz[k] * esize);
  const int counts[5] = {p->n_sources, p->n_ports, p->n_mx, p->n_my, p->n_probes};
  for (int k = 0; k < 5; ++k) {
    L.off[k] = cv.take<int>(L.n_tiles + 1);
    L.pts[k] = cv.take<int2>(std::max(counts[k], 1));
  }
  L.step = cv.take<int>(1);
  L.eacc = cv.take<double>(p->record_energy ? 2 * size_t(std::max(p->n_steps, 1)) : 1);
  L.total = cv.bytes();
  return L;
}

static int validate(const GdnTmParams* p, const GdnTmPoints* pts, const GdnTmBuffers* b) {
  if (!p || !pts || !b) GDN_BAD_ARG("null params/points/buffers");
  const int nx = p->nx, ny = p->ny;
  if (nx < 3 || ny < 3) GDN_BAD_ARG("grid must be at least 3x3, got %dx%d", nx, ny);
  if (p->npml < 0) GDN_BAD_ARG("npml must be >= 0");
  if (std::min(nx, ny) <= 2 * p->npml + 2)
    GDN_BAD_ARG("grid %dx%d is too small for CPML thickness %d", nx, ny, p->npml);
  if (p->n_steps < 0) GDN_BAD_ARG("n_steps must be >= 0");
  if (p->n_sources < 0 || p->n_ports < 0 || p->n_mx < 0 || p->n_my < 0 || p->n_probes < 0 ||
      p->n_freq < 0)
    GDN_BAD_ARG("negative count");
  if (p->n_freq > KMAX) GDN_BAD_ARG("n_freq %d exceeds the supported maximum %d", p->n_freq, KMAX);
  if ((long long)nx * ny > (1LL << 31) / 4) GDN_BAD_ARG("grid too large for 32-bit cell ids");
  auto check = [&](int n, const int32_t* a, const int32_t* bb, int lo_i, int hi_i, int lo_j,
                   int hi_j, const char* name) -> int {
    if (n > 0 && (!a || !bb)) GDN_BAD_ARG("%s index arrays are null", name);
    for (int m = 0; m < n; ++m)
      if (a[m] < lo_i || a[m] > hi_i || bb[m] < lo_j || bb[m] > hi_j)
        GDN_BAD_ARG("%s index (%d, %d) outside [%d..%d] x [%d..%d]", name, a[m], bb[m], lo_i,
                    hi_i, lo_j, hi_j);
    return GDN_OK;
  };
  int s;
  if ((s = check(p->n_sources, pts->src_i, pts->src_j, 1, nx - 2, 1, ny - 2, "source_ij"))) return s;
  if ((s = check(p->n_ports, pts->port_i, pts->port_j, 1, nx - 2, 1, ny - 2, "port ij"))) return s;
  if ((s = check(p->n_mx, pts->mx_i, pts->mx_j, 0, nx - 1, 0, ny - 2, "mx_ij"))) return s;
  if ((s = check(p->n_my, pts->my_i, pts->my_j, 0, nx - 2, 0, ny - 1, "my_ij"))) return s;
  if ((s = check(p->n_probes, pts->probe_i, pts->probe_j, 0, nx - 1, 0, ny - 1, "probe_ij")))
    return s;
  if (!b->ca || !b->cb) GDN_BAD_ARG("ca/cb are null");
  if (!b->inv_kx_e || !b->inv_ky_e || !b->inv_kx_h || !b->inv_ky_h)
    GDN_BAD_ARG("1/kappa tables are null");
  if (p->npml > 0) {
    const void* t[16] = {b->b_ezx_lo, b->c_ezx_lo, b->b_ezx_hi, b->c_ezx_hi, b->b_ezy_lo, b->c_ezy_lo,
                         b->b_ezy_hi, b->c_ezy_hi, b->b_hyx_lo, b->c_hyx_lo, b->b_hyx_hi, b->c_hyx_hi,
                         b->b_hxy_lo, b->c_hxy_lo, b->b_hxy_hi, b->c_hxy_hi};
    for (auto x : t)
      if (!x) GDN_BAD_ARG("a CPML slab table is null");
  }
  if (!b->ez || !b->hx || !b->hy) GDN_BAD_ARG("output field buffers are null");
  if (p->n_probes > 0 && p->n_steps > 0 && !b->out_probe) GDN_BAD_ARG("out_probe is null");
  const bool steps = p->n_steps > 0;  // zero-step runs touch no per-step array
  if (p->n_ports > 0 && steps && (!b->out_v || !b->out_i || !b->cb_vs || !b->port_vs))
    GDN_BAD_ARG("port buffers are null");
  if (p->record_energy && steps && (!b->out_energy || !b->eps))
    GDN_BAD_ARG("energy buffers are null");
  if (p->n_freq > 0 && steps && (!b->ph_e || !b->ph_h)) GDN_BAD_ARG("phase tables are null");
  if (p->cw_sources) {
    if (p->n_freq <= 0) GDN_BAD_ARG("cw_sources needs n_freq > 0");
    if (!b->cw_env) GDN_BAD_ARG("cw_env is null");
    if ((p->n_sources && !b->src_w) || (p->n_mx && !b->mx_w) || (p->n_my && !b->my_w))
      GDN_BAD_ARG("cw weight arrays are null");
  } else if (steps) {
    if ((p->n_sources && !b->src_cur) || (p->n_mx && !b->mx_cur) || (p->n_my && !b->my_cur))
      GDN_BAD_ARG("source waveform arrays are null");
  }
  if (p->n_sources && !b->cb_src) GDN_BAD_ARG("cb_src is null");
  if (p->n_freq > 0) {
    if (!b->dft_ez || !b->dft_hx || !b->dft_hy) {
      if (!p->use_dft_region) GDN_BAD_ARG("dft output buffers are null");
    }
    if (p->use_dft_region) {
      const int shp[3][2] = {{nx, ny}, {nx, ny - 1}, {nx - 1, ny}};
      void* const outs[3] = {b->dft_ez, b->dft_hx, b->dft_hy};
      for (int c = 0; c < 3; ++c) {
        const int* lo = p->dft_lo[c];
        const int* hi = p->dft_hi[c];
        if (hi[0] <= lo[0] || hi[1] <= lo[1]) continue;
        if (lo[0] < 0 || lo[1] < 0 || hi[0] > shp[c][0] || hi[1] > shp[c][1])
          GDN_BAD_ARG("dft region %d [%d,%d)x[%d,%d) outside its component", c, lo[0], hi[0],
                      lo[1], hi[1]);
        if (!outs[c]) GDN_BAD_ARG("dft output %d is null", c);
      }
    }
  }
  if (p->dt <= 0 || p->dx <= 0 || p->dy <= 0) GDN_BAD_ARG("dt, dx, dy must be positive");
  return GDN_OK;
}

template <typename T>
static int run(const GdnTmParams* p, const GdnTmPoints* pts, const GdnTmBuffers* b,
               cudaStream_t stream) {
  using A_f = float;
  int st = validate(p, pts, b);
  if (st) return st;
  const Layout L = make_layout(p, sizeof(T));
  char* ws = static_cast<char*>(b->workspace);
  bool own = false;
  if (!ws) {
    GDN_TRY_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ws), L.total, stream));
    own = true;
  } else if (b->workspace_bytes < L.total) {
    GDN_BAD_ARG("workspace too small: %zu < %zu bytes", b->workspace_bytes, L.total);
  }
  struct Guard {
    char* p;
    bool own;
    cudaStream_t s;
    ~Guard() {
      if (own && p) cudaFreeAsync(p, s);
    }
  } guard{ws, own, stream};

  const int nx = p->nx, ny = p->ny, N = p->n_steps;
  Dev<T> d{};
  d.nx = nx;
  d.ny = ny;
  d.ld = L.ld;
  d.npml = p->npml;
  d.R = L.R;
  d.n_steps = N;
  d.n_freq = p->n_freq;
  d.tiles_x = L.tiles_x;
  d.slot = L.slot;
  d.ring = reinterpret_cast<T*>(ws + L.ring);
  d.ca = static_cast<const T*>(b->ca);
  d.cb = static_cast<const T*>(b->cb);
  d.eps = static_cast<const T*>(b->eps);
  d.ikx_e = static_cast<const T*>(b->inv_kx_e);
  d.iky_e = static_cast<const T*>(b->inv_ky_e);
  d.ikx_h = static_cast<const T*>(b->inv_kx_h);
  d.iky_h = static_cast<const T*>(b->inv_ky_h);
#define GDN_TAB(x) d.x = static_cast<const T*>(b->x)
  GDN_TAB(b_ezx_lo); GDN_TAB(c_ezx_lo); GDN_TAB(b_ezx_hi); GDN_TAB(c_ezx_hi);
  GDN_TAB(b_ezy_lo); GDN_TAB(c_ezy_lo); GDN_TAB(b_ezy_hi); GDN_TAB(c_ezy_hi);
  GDN_TAB(b_hyx_lo); GDN_TAB(c_hyx_lo); GDN_TAB(b_hyx_hi); GDN_TAB(c_hyx_hi);
  GDN_TAB(b_hxy_lo); GDN_TAB(c_hxy_lo); GDN_TAB(b_hxy_hi); GDN_TAB(c_hxy_hi);
#undef GDN_TAB
  T* psi[8];
  for (int k = 0; k < 8; ++k) psi[k] = reinterpret_cast<T*>(ws + L.psi[k]);
  d.ezx_lo = psi[0]; d.ezx_hi = psi[1]; d.ezy_lo = psi[2]; d.ezy_hi = psi[3];
  d.hyx_lo = psi[4]; d.hyx_hi = psi[5]; d.hxy_lo = psi[6]; d.hxy_hi = psi[7];
  d.dt_mu = T(b->dt_mu);
  d.inv_dx = T(b->inv_dx);
  d.inv_dy = T(b->inv_dy);
  d.dx = T(p->dx);
  d.dy = T(p->dy);
  d.dz = T(p->dz);
  d.n_src = p->n_sources;
  d.n_ports = p->n_ports;
  d.n_mx = p->n_mx;
  d.n_my = p->n_my;
  d.n_probes = p->n_probes;
  d.cb_src = static_cast<const T*>(b->cb_src);
  d.src_cur = static_cast<const T*>(b->src_cur);
  d.cb_vs = static_cast<const T*>(b->cb_vs);
  d.port_vs = static_cast<const T*>(b->port_vs);
  d.mx_cur = static_cast<const T*>(b->mx_cur);
  d.my_cur = static_cast<const T*>(b->my_cur);
  d.cw = p->cw_sources;
  d.cw_env = b->cw_env;
  d.src_w = reinterpret_cast<const double2*>(b->src_w);
  d.mx_w = reinterpret_cast<const double2*>(b->mx_w);
  d.my_w = reinterpret_cast<const double2*>(b->my_w);
  d.ph_e = reinterpret_cast<const double2*>(b->ph_e);
  d.ph_h = reinterpret_cast<const double2*>(b->ph_h);
  d.out_probe = static_cast<T*>(b->out_probe);
  d.out_v = static_cast<T*>(b->out_v);
  d.out_i = static_cast<T*>(b->out_i);
  int* step_base = reinterpret_cast<int*>(ws + L.step);
  d.step_base = step_base;

  // Bin the point lists by tile and upload them.
  const int counts[5] = {p->n_sources, p->n_ports, p->n_mx, p->n_my, p->n_probes};
  const int32_t* is[5] = {pts->src_i, pts->port_i, pts->mx_i, pts->my_i, pts->probe_i};
  const int32_t* js[5] = {pts->src_j, pts->port_j, pts->mx_j, pts->my_j, pts->probe_j};
  const int* offs[5];
  const int2* pls[5];
  for (int k = 0; k < 5; ++k) {
    PointBins pb = bin_points(counts[k], is[k], js[k], TI, TJ, L.tiles_x, L.n_tiles, L.ld);
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.off[k], pb.off.data(), pb.off.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    if (counts[k] > 0)
      GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.pts[k], pb.pts.data(), pb.pts.size() * sizeof(int2),
                                   cudaMemcpyHostToDevice, stream));
    offs[k] = reinterpret_cast<const int*>(ws + L.off[k]);
    pls[k] = reinterpret_cast<const int2*>(ws + L.pts[k]);
  }
  // Pageable host vectors above are staged by the copy before it returns.
  d.src_off = offs[0]; d.src_pts = pls[0];
  d.port_off = offs[1]; d.port_pts = pls[1];
  d.mx_off = offs[2]; d.mx_pts = pls[2];
  d.my_off = offs[3]; d.my_pts = pls[3];
  d.probe_off = offs[4]; d.probe_pts = pls[4];

  // Zero the state: ring, psi, counter, energy accumulators, DFT outputs.
  GDN_TRY_CUDA(cudaMemsetAsync(ws + L.ring, 0, size_t(L.R) * L.slot * sizeof(T), stream));
  // The eight psi slabs are carved back to back, ending where off[0] starts.
  GDN_TRY_CUDA(cudaMemsetAsync(ws + L.psi[0], 0, L.off[0] - L.psi[0], stream));
  GDN_TRY_CUDA(cudaMemsetAsync(step_base, 0, sizeof(int), stream));
  double* eacc = reinterpret_cast<double*>(ws + L.eacc);
  if (p->record_energy)
    GDN_TRY_CUDA(cudaMemsetAsync(eacc, 0, 2 * size_t(std::max(N, 1)) * sizeof(double), stream));

  const bool f64acc = p->dft_f64 != 0;
  const size_t csz = f64acc ? sizeof(double2) : sizeof(float2);
  DftDev<float> qf{};
  DftDev<double> qd{};
  long long dft_counts[3] = {0, 0, 0};
  void* const dft_out[3] = {b->dft_ez, b->dft_hx, b->dft_hy};
  const int full_shape[3][2] = {{nx, ny}, {nx, ny - 1}, {nx - 1, ny}};
  for (int c = 0; c < 3; ++c) {
    int lo0 = 0, lo1 = 0, hi0 = full_shape[c][0], hi1 = full_shape[c][1];
    if (p->use_dft_region) {
      lo0 = p->dft_lo[c][0]; lo1 = p->dft_lo[c][1];
      hi0 = p->dft_hi[c][0]; hi1 = p->dft_hi[c][1];
      if (hi0 <= lo0 || hi1 <= lo1) { lo0 = lo1 = hi0 = hi1 = 0; }
    }
    if (p->n_freq == 0) { lo0 = lo1 = hi0 = hi1 = 0; }
    qf.lo[c][0] = qd.lo[c][0] = lo0; qf.lo[c][1] = qd.lo[c][1] = lo1;
    qf.hi[c][0] = qd.hi[c][0] = hi0; qf.hi[c][1] = qd.hi[c][1] = hi1;
    qf.acc[c] = static_cast<float2*>(dft_out[c]);
    qd.acc[c] = static_cast<double2*>(dft_out[c]);
    dft_counts[c] = (long long)(hi0 - lo0) * (hi1 - lo1);
    if (dft_counts[c] > 0)
      GDN_TRY_CUDA(cudaMemsetAsync(dft_out[c], 0, size_t(dft_counts[c]) * p->n_freq * csz, stream));
  }
  const long long max_cells = std::max({dft_counts[0], dft_counts[1], dft_counts[2]});

  const dim3 blk(TJ, TI);
  const dim3 grd(L.tiles_x, L.tiles_y);
  const int eblocks = int(std::min<long long>(div_up((long long)nx * ny, 256), 148 * 8));

  // Capture one chunk of `cnt` steps as a graph.
  auto capture = [&](int cnt, cudaGraphExec_t* exec) -> int {
    cudaStream_t cs = capture_stream();
    if (!cs) GDN_BAD_ARG("no capture stream for this device");
    GDN_TRY_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < cnt; ++s) {
      tm_h_sweep<T><<<grd, blk, 0, cs>>>(d, s);
      tm_e_sweep<T><<<grd, blk, 0, cs>>>(d, s);
      if (p->record_energy) tm_energy<T><<<eblocks, 256, 0, cs>>>(d, eacc, s);
    }
    if (p->n_freq > 0 && max_cells > 0) {
      const dim3 dg(unsigned(div_up(max_cells, 256)), 3);
      if (f64acc) {
        const size_t sm = size_t(4) * cnt * p->n_freq * sizeof(double);
        tm_dft_fold<T, double><<<dg, 256, sm, cs>>>(d, qd, 0, cnt);
      } else {
        const size_t sm = size_t(4) * cnt * p->n_freq * sizeof(float);
        tm_dft_fold<T, A_f><<<dg, 256, sm, cs>>>(d, qf, 0, cnt);
      }
    }
    tm_advance<<<1, 1, 0, cs>>>(step_base, cnt);
    cudaGraph_t g = nullptr;
    cudaError_t e1 = cudaStreamEndCapture(cs, &g);
    if (e1 != cudaSuccess) {
      set_error("graph capture failed: %s", cudaGetErrorString(e1));
      return GDN_ERR_CUDA;
    }
    cudaError_t e2 = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
      set_error("graph instantiate failed: %s", cudaGetErrorString(e2));
      return GDN_ERR_CUDA;
    }
    return GDN_OK;
  };

  const int Tc = L.T;
  const int full = N / Tc, rem = N % Tc;
  cudaGraphExec_t g_full = nullptr, g_rem = nullptr;
  if (full > 0 && (st = capture(Tc, &g_full))) return st;
  if (rem > 0 && (st = capture(rem, &g_rem))) {
    if (g_full) cudaGraphExecDestroy(g_full);
    return st;
  }
  cudaError_t le = cudaSuccess;
  for (int c = 0; c < full && le == cudaSuccess; ++c) le = cudaGraphLaunch(g_full, stream);
  if (rem > 0 && le == cudaSuccess) le = cudaGraphLaunch(g_rem, stream);
  if (g_full) cudaGraphExecDestroy(g_full);
  if (g_rem) cudaGraphExecDestroy(g_rem);
  if (le != cudaSuccess) {
    set_error("graph launch failed: %s", cudaGetErrorString(le));
    return GDN_ERR_CUDA;
  }

  // Finalise: fields out, DFT x dt (fdtd2d.py:482-487), energy.
  const T* last = d.ring + (long long)(N % L.R) * L.slot;
  tm_copy_out<T><<<eblocks, 256, 0, stream>>>(last, nx, ny, L.ld, static_cast<T*>(b->ez),
                                                  static_cast<T*>(b->hx), static_cast<T*>(b->hy));
  for (int c = 0; c < 3; ++c) {
    if (dft_counts[c] <= 0 || p->n_freq == 0) continue;
    const long long cnt = dft_counts[c] * p->n_freq;
    const int blocks = int(std::min<long long>(div_up(cnt, 256), 148 * 8));
    if (f64acc)
      tm_dft_scale<double2><<<blocks, 256, 0, stream>>>(static_cast<double2*>(dft_out[c]), cnt, p->dt);
    else
      tm_dft_scale<float2><<<blocks, 256, 0, stream>>>(static_cast<float2*>(dft_out[c]), cnt, p->dt);
  }
  if (p->record_energy && N > 0)
    tm_energy_finish<T><<<unsigned(div_up(N, 256)), 256, 0, stream>>>(
        eacc, static_cast<T*>(b->out_energy), N, p->dx * p->dy, p->mu0);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

}  // namespace tm2d
}  // namespace gdn

extern "C" int gdn_tm_workspace_size(const GdnTmParams* p, int f64, size_t* bytes) {
  if (!p || !bytes) {
    gdn::set_error("null argument");
    return GDN_ERR_BAD_ARG;
  }
  if (p->nx < 3 || p->ny < 3 || p->npml < 0) {
    gdn::set_error("invalid grid");
    return GDN_ERR_BAD_ARG;
  }
  *bytes = gdn::tm2d::make_layout(p, f64 ? sizeof(double) : sizeof(float)).total;
  return GDN_OK;
}

extern "C" int gdn_tm_run_f32(const GdnTmParams* p, const GdnTmPoints* pts,
                              const GdnTmBuffers* b, void* stream) {
  return gdn::tm2d::run<float>(p, pts, b, static_cast<cudaStream_t>(stream));
}

extern "C" int gdn_tm_run_f64(const GdnTmParams* p, const GdnTmPoints* pts,
                              const GdnTmBuffers* b, void* stream) {
  return gdn::tm2d::run<double>(p, pts, b, static_cast<cudaStream_t>(stream));
}
