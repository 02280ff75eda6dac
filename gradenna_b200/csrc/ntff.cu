// Near-to-far-field projection kernels (3D box and 2D contour).
//
//   gdn_ntff3d_project       ntff_3d radiation vectors -> E_theta, E_phi
//                            (src/gradenna/ntff.py:399-428)
//   gdn_ntff3d_project_grad  its adjoint (the map is complex-linear in J, M)
//   gdn_ntff2d_project       ntff_2d contour integral (ntff.py:213-228)
//
// The work is n_freq x n_dir x n_pts complex exponentials with a dozen
// complex multiply-adds each. One CTA owns a tile of DPT directions at one
// frequency; its threads stride over the surface points, so each point's
// position and currents are read once per tile, the phase of every
// direction is formed in registers, and the partial radiation vectors are
// reduced with warp shuffles and shared memory. Precision follows the
// phasor type: float math for complex64, double for complex128.
#include "common.cuh"

namespace gdn {
namespace ntff {

template <typename A>
struct CT;
template <>
struct CT<float> {
  using C = float2;
};
template <>
struct CT<double> {
  using C = double2;
};

template <typename A>
__device__ __forceinline__ void sc(A x, A* s, A* c);
template <>
__device__ __forceinline__ void sc<float>(float x, float* s, float* c) {
  sincosf(x, s, c);
}
template <>
__device__ __forceinline__ void sc<double>(double x, double* s, double* c) {
  sincos(x, s, c);
}

template <typename A>
__device__ __forceinline__ A warp_sum(A v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

constexpr int NT = 256;

// Block-wide sum of `nv` per-thread values; result valid in thread 0.
template <typename A, int NV>
__device__ __forceinline__ void block_sum(A (&v)[NV], A* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    const A s = warp_sum(v[q]);
    if (lane == 0) red[wid * NV + q] = s;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    A s = 0;
    for (int w = 0; w < NT / 32; ++w) s += red[w * NV + threadIdx.x];
    red[threadIdx.x] = s;  // reads of this column are done by this thread only
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = red[q];
}

template <typename A, int DPT>
__global__ void __launch_bounds__(NT) ntff3d_kernel(int n_pts, int n_dir, const double* pos,
                                                    const double* w,
                                                    const typename CT<A>::C* J,
                                                    const typename CT<A>::C* M, const double* kw,
                                                    const double* dirs, double eta0,
                                                    typename CT<A>::C* out) {
  using C = typename CT<A>::C;
  constexpr int NV = DPT * 12;
  __shared__ A red[(NT / 32) * NV];
  const int f = blockIdx.y;
  const int d0 = blockIdx.x * DPT;
  const A k = A(kw[f]);
  A rx[DPT], ry[DPT], rz[DPT];
#pragma unroll
  for (int q = 0; q < DPT; ++q) {
    const int d = min(d0 + q, n_dir - 1);
    const A ct = A(dirs[4 * d]), st = A(dirs[4 * d + 1]), cp = A(dirs[4 * d + 2]),
            sp = A(dirs[4 * d + 3]);
    rx[q] = st * cp;
    ry[q] = st * sp;
    rz[q] = ct;
  }
  A acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = A(0);
  const C* Jf = J + (long long)f * n_pts * 3;
  const C* Mf = M + (long long)f * n_pts * 3;
  for (int p = threadIdx.x; p < n_pts; p += NT) {
    const A x = A(pos[3 * p]), y = A(pos[3 * p + 1]), z = A(pos[3 * p + 2]);
    const A wp = A(w[p]);
    C j3[3], m3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      j3[c] = Jf[3 * p + c];
      m3[c] = Mf[3 * p + c];
    }
#pragma unroll
    for (int q = 0; q < DPT; ++q) {
      A s, cc;
      sc<A>(k * (x * rx[q] + y * ry[q] + z * rz[q]), &s, &cc);
      const A pr = wp * cc, pi = wp * s;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc[q * 12 + 2 * c] += pr * j3[c].x - pi * j3[c].y;
        acc[q * 12 + 2 * c + 1] += pr * j3[c].y + pi * j3[c].x;
        acc[q * 12 + 6 + 2 * c] += pr * m3[c].x - pi * m3[c].y;
        acc[q * 12 + 6 + 2 * c + 1] += pr * m3[c].y + pi * m3[c].x;
      }
    }
  }
  block_sum<A, NV>(acc, red);
  if (threadIdx.x < DPT && d0 + threadIdx.x < n_dir) {
    const int q = threadIdx.x, d = d0 + q;
    const A ct = A(dirs[4 * d]), st = A(dirs[4 * d + 1]), cp = A(dirs[4 * d + 2]),
            sp = A(dirs[4 * d + 3]);
    const A* a = acc + q * 12;
    // N_theta, N_phi, L_theta, L_phi (re, im)
    const A nth_r = (a[0] * cp + a[2] * sp) * ct - a[4] * st;
    const A nth_i = (a[1] * cp + a[3] * sp) * ct - a[5] * st;
    const A nph_r = -a[0] * sp + a[2] * cp, nph_i = -a[1] * sp + a[3] * cp;
    const A lth_r = (a[6] * cp + a[8] * sp) * ct - a[10] * st;
    const A lth_i = (a[7] * cp + a[9] * sp) * ct - a[11] * st;
    const A lph_r = -a[6] * sp + a[8] * cp, lph_i = -a[7] * sp + a[9] * cp;
    const A cf = k / A(4.0 * 3.14159265358979323846);  // coef = i cf
    const A e0 = A(eta0);
    // E_theta = -i cf (L_phi + eta0 N_theta); E_phi = i cf (L_theta - eta0 N_phi)
    const A ur = lph_r + e0 * nth_r, ui = lph_i + e0 * nth_i;
    const A vr = lth_r - e0 * nph_r, vi = lth_i - e0 * nph_i;
    C eth, eph;
    eth.x = cf * ui;
    eth.y = -cf * ur;
    eph.x = -cf * vi;
    eph.y = cf * vr;
    out[((long long)f * n_dir + d) * 2] = eth;
    out[((long long)f * n_dir + d) * 2 + 1] = eph;
  }
}

// Adjoint: per point, g_J = sum_d conj(ph_dp) g_N_d, g_M = sum_d conj(ph_dp) g_L_d,
// with g_N / g_L from g_out through the conjugate of the theta/phi map.
template <typename A>
__global__ void __launch_bounds__(NT) ntff3d_grad_kernel(int n_pts, int n_dir, const double* pos,
                                                         const double* w, const double* kw,
                                                         const double* dirs, double eta0,
                                                         const typename CT<A>::C* g_out,
                                                         typename CT<A>::C* gJ,
                                                         typename CT<A>::C* gM) {
  using C = typename CT<A>::C;
  constexpr int DCH = 64;  // directions staged per round
  __shared__ A s_r[DCH][3];
  __shared__ A s_g[DCH][12];  // g_N (x,y,z re/im), g_L (x,y,z re/im)
  const int f = blockIdx.y;
  const int p = blockIdx.x * NT + threadIdx.x;
  const A k = A(kw[f]);
  const A cf = k / A(4.0 * 3.14159265358979323846);
  const A e0 = A(eta0);
  A x = 0, y = 0, z = 0, wp = 0;
  if (p < n_pts) {
    x = A(pos[3 * p]);
    y = A(pos[3 * p + 1]);
    z = A(pos[3 * p + 2]);
    wp = A(w[p]);
  }
  A aj[6] = {0, 0, 0, 0, 0, 0}, am[6] = {0, 0, 0, 0, 0, 0};
  for (int base = 0; base < n_dir; base += DCH) {
    __syncthreads();
    for (int q = threadIdx.x; q < DCH; q += NT) {
      const int d = base + q;
      if (d >= n_dir) break;
      const A ct = A(dirs[4 * d]), st = A(dirs[4 * d + 1]), cp = A(dirs[4 * d + 2]),
              sp = A(dirs[4 * d + 3]);
      s_r[q][0] = st * cp;
      s_r[q][1] = st * sp;
      s_r[q][2] = ct;
      const C gt = g_out[((long long)f * n_dir + d) * 2];
      const C gp = g_out[((long long)f * n_dir + d) * 2 + 1];
      // conj(-i cf) = i cf, conj(i cf) = -i cf:
      // g_Lph = i cf gt, g_Nth = i cf eta0 gt, g_Lth = -i cf gp, g_Nph = i cf eta0 gp
      const A lph_r = -cf * gt.y, lph_i = cf * gt.x;
      const A nth_r = e0 * lph_r, nth_i = e0 * lph_i;
      const A lth_r = cf * gp.y, lth_i = -cf * gp.x;
      const A nph_r = -e0 * cf * gp.y, nph_i = e0 * cf * gp.x;
      // back through N_theta = (Nx cp + Ny sp) ct - Nz st, N_phi = -Nx sp + Ny cp
      s_g[q][0] = cp * ct * nth_r - sp * nph_r;
      s_g[q][1] = cp * ct * nth_i - sp * nph_i;
      s_g[q][2] = sp * ct * nth_r + cp * nph_r;
      s_g[q][3] = sp * ct * nth_i + cp * nph_i;
      s_g[q][4] = -st * nth_r;
      s_g[q][5] = -st * nth_i;
      s_g[q][6] = cp * ct * lth_r - sp * lph_r;
      s_g[q][7] = cp * ct * lth_i - sp * lph_i;
      s_g[q][8] = sp * ct * lth_r + cp * lph_r;
      s_g[q][9] = sp * ct * lth_i + cp * lph_i;
      s_g[q][10] = -st * lth_r;
      s_g[q][11] = -st * lth_i;
    }
    __syncthreads();
    const int nd = min(DCH, n_dir - base);
    if (p < n_pts) {
      for (int q = 0; q < nd; ++q) {
        A s, c;
        sc<A>(k * (x * s_r[q][0] + y * s_r[q][1] + z * s_r[q][2]), &s, &c);
        const A pr = wp * c, pi = -wp * s;  // conj(phase)
#pragma unroll
        for (int cpn = 0; cpn < 3; ++cpn) {
          aj[2 * cpn] += pr * s_g[q][2 * cpn] - pi * s_g[q][2 * cpn + 1];
          aj[2 * cpn + 1] += pr * s_g[q][2 * cpn + 1] + pi * s_g[q][2 * cpn];
          am[2 * cpn] += pr * s_g[q][6 + 2 * cpn] - pi * s_g[q][6 + 2 * cpn + 1];
          am[2 * cpn + 1] += pr * s_g[q][6 + 2 * cpn + 1] + pi * s_g[q][6 + 2 * cpn];
        }
      }
    }
  }
  if (p < n_pts) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      C vj, vm;
      vj.x = aj[2 * c];
      vj.y = aj[2 * c + 1];
      vm.x = am[2 * c];
      vm.y = am[2 * c + 1];
      gJ[((long long)f * n_pts + p) * 3 + c] = vj;
      gM[((long long)f * n_pts + p) * 3 + c] = vm;
    }
  }
}

template <typename A, int DPT>
__global__ void __launch_bounds__(NT) ntff2d_kernel(int n_pts, int n_ang, const double* pos,
                                                    const double* w,
                                                    const typename CT<A>::C* Jz,
                                                    const typename CT<A>::C* Ez, const double* kw,
                                                    const double* ang, double eta0,
                                                    typename CT<A>::C* out) {
  using C = typename CT<A>::C;
  __shared__ A red[(NT / 32) * DPT * 2];
  const int f = blockIdx.y;
  const int a0 = blockIdx.x * DPT;
  const A k = A(kw[f]);
  A ca[DPT], sa[DPT], acc[DPT * 2];
#pragma unroll
  for (int q = 0; q < DPT; ++q) {
    const int a = min(a0 + q, n_ang - 1);
    double s, c;
    sincos(ang[a], &s, &c);
    sa[q] = A(s);
    ca[q] = A(c);
    acc[2 * q] = acc[2 * q + 1] = A(0);
  }
  const A e0 = A(eta0);
  for (int p = threadIdx.x; p < n_pts; p += NT) {
    const A x = A(pos[4 * p]), y = A(pos[4 * p + 1]), nx = A(pos[4 * p + 2]),
            ny = A(pos[4 * p + 3]);
    const A wp = A(w[p]);
    const C j = Jz[(long long)f * n_pts + p], e = Ez[(long long)f * n_pts + p];
#pragma unroll
    for (int q = 0; q < DPT; ++q) {
      const A md = nx * ca[q] + ny * sa[q];
      const A ir = e0 * j.x - md * e.x, ii = e0 * j.y - md * e.y;
      A s, c;
      sc<A>(k * (x * ca[q] + y * sa[q]), &s, &c);
      acc[2 * q] += wp * (c * ir - s * ii);
      acc[2 * q + 1] += wp * (c * ii + s * ir);
    }
  }
  block_sum<A, DPT * 2>(acc, red);
  if (threadIdx.x < DPT && a0 + threadIdx.x < n_ang) {
    const int q = threadIdx.x;
    // prefactor -sqrt(i k / 8 pi) = -sqrt(k / 8 pi) (1 + i) / sqrt(2)
    const A m = -sqrt(k / A(8.0 * 3.14159265358979323846)) / sqrt(A(2));
    C o;
    o.x = m * (acc[2 * q] - acc[2 * q + 1]);
    o.y = m * (acc[2 * q] + acc[2 * q + 1]);
    out[(long long)f * n_ang + a0 + q] = o;
  }
}

// Adjoint of the 2D projection: per point, g_Jz = sum_a conj(a_Jz) g_a and
// g_Ez = sum_a conj(a_Ez) g_a with a_Jz = pref w eta0 ph, a_Ez = -pref w (n.u) ph.
template <typename A>
__global__ void __launch_bounds__(NT) ntff2d_grad_kernel(int n_pts, int n_ang, const double* pos,
                                                         const double* w, const double* kw,
                                                         const double* ang, double eta0,
                                                         const typename CT<A>::C* g_out,
                                                         typename CT<A>::C* gJ,
                                                         typename CT<A>::C* gE) {
  using C = typename CT<A>::C;
  constexpr int ACH = 128;
  __shared__ A s_c[ACH], s_s[ACH], s_g[ACH][2];
  const int f = blockIdx.y;
  const int p = blockIdx.x * NT + threadIdx.x;
  const A k = A(kw[f]);
  // conj(pref) = -sqrt(k / 8 pi)(1 - i)/sqrt(2)
  const A m = -sqrt(k / A(8.0 * 3.14159265358979323846)) / sqrt(A(2));
  A x = 0, y = 0, nx = 0, ny = 0, wp = 0;
  if (p < n_pts) {
    x = A(pos[4 * p]);
    y = A(pos[4 * p + 1]);
    nx = A(pos[4 * p + 2]);
    ny = A(pos[4 * p + 3]);
    wp = A(w[p]);
  }
  A sr = 0, si = 0, tr = 0, ti = 0;  // sum conj(ph) g,  sum (n.u) conj(ph) g
  for (int base = 0; base < n_ang; base += ACH) {
    __syncthreads();
    for (int q = threadIdx.x; q < ACH; q += NT) {
      const int a = base + q;
      if (a >= n_ang) break;
      double s, c;
      sincos(ang[a], &s, &c);
      s_c[q] = A(c);
      s_s[q] = A(s);
      const C g = g_out[(long long)f * n_ang + a];
      s_g[q][0] = g.x;
      s_g[q][1] = g.y;
    }
    __syncthreads();
    const int na = min(ACH, n_ang - base);
    if (p < n_pts) {
      for (int q = 0; q < na; ++q) {
        A s, c;
        sc<A>(k * (x * s_c[q] + y * s_s[q]), &s, &c);
        const A gr = s_g[q][0], gi = s_g[q][1];
        const A vr = c * gr + s * gi, vi = c * gi - s * gr;  // conj(ph) g
        const A md = nx * s_c[q] + ny * s_s[q];
        sr += vr;
        si += vi;
        tr += md * vr;
        ti += md * vi;
      }
    }
  }
  if (p < n_pts) {
    // conj(pref) (a + i b) = m ((a + b) + i (b - a))
    const A e0 = A(eta0);
    C vj, ve;
    vj.x = wp * e0 * m * (sr + si);
    vj.y = wp * e0 * m * (si - sr);
    ve.x = -wp * m * (tr + ti);
    ve.y = -wp * m * (ti - tr);
    gJ[(long long)f * n_pts + p] = vj;
    gE[(long long)f * n_pts + p] = ve;
  }
}

}  // namespace ntff
}  // namespace gdn

using namespace gdn::ntff;

extern "C" int gdn_ntff3d_project(int32_t n_freq, int32_t n_pts, int32_t n_dir, int32_t c128,
                                  const double* pos, const double* w, const void* J,
                                  const void* M, const double* k, const double* dirs,
                                  double eta0, void* out, void* stream) {
  if (n_freq < 0 || n_pts < 0 || n_dir < 0) GDN_BAD_ARG("negative size");
  if (n_freq == 0 || n_dir == 0) return GDN_OK;
  if (!pos || !w || !J || !M || !k || !dirs || !out) GDN_BAD_ARG("null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (c128) {
    constexpr int D = 2;
    ntff3d_kernel<double, D><<<dim3(unsigned(gdn::div_up(n_dir, D)), n_freq), NT, 0, s>>>(
        n_pts, n_dir, pos, w, static_cast<const double2*>(J), static_cast<const double2*>(M), k,
        dirs, eta0, static_cast<double2*>(out));
  } else {
    constexpr int D = 4;
    ntff3d_kernel<float, D><<<dim3(unsigned(gdn::div_up(n_dir, D)), n_freq), NT, 0, s>>>(
        n_pts, n_dir, pos, w, static_cast<const float2*>(J), static_cast<const float2*>(M), k,
        dirs, eta0, static_cast<float2*>(out));
  }
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_ntff3d_project_grad(int32_t n_freq, int32_t n_pts, int32_t n_dir,
                                       int32_t c128, const double* pos, const double* w,
                                       const double* k, const double* dirs, double eta0,
                                       const void* g_out, void* g_J, void* g_M, void* stream) {
  if (n_freq < 0 || n_pts < 0 || n_dir < 0) GDN_BAD_ARG("negative size");
  if (n_freq == 0 || n_pts == 0) return GDN_OK;
  if (!pos || !w || !k || !dirs || !g_out || !g_J || !g_M) GDN_BAD_ARG("null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid(unsigned(gdn::div_up(n_pts, NT)), n_freq);
  if (c128)
    ntff3d_grad_kernel<double><<<grid, NT, 0, s>>>(n_pts, n_dir, pos, w, k, dirs, eta0,
                                                   static_cast<const double2*>(g_out),
                                                   static_cast<double2*>(g_J),
                                                   static_cast<double2*>(g_M));
  else
    ntff3d_grad_kernel<float><<<grid, NT, 0, s>>>(n_pts, n_dir, pos, w, k, dirs, eta0,
                                                  static_cast<const float2*>(g_out),
                                                  static_cast<float2*>(g_J),
                                                  static_cast<float2*>(g_M));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_ntff2d_project(int32_t n_freq, int32_t n_pts, int32_t n_ang, int32_t c128,
                                  const double* pos, const double* w, const void* Jz,
                                  const void* Ez, const double* k, const double* angles,
                                  double eta0, void* out, void* stream) {
  if (n_freq < 0 || n_pts < 0 || n_ang < 0) GDN_BAD_ARG("negative size");
  if (n_freq == 0 || n_ang == 0) return GDN_OK;
  if (!pos || !w || !Jz || !Ez || !k || !angles || !out) GDN_BAD_ARG("null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  constexpr int D = 4;
  const dim3 grid(unsigned(gdn::div_up(n_ang, D)), n_freq);
  if (c128)
    ntff2d_kernel<double, D><<<grid, NT, 0, s>>>(n_pts, n_ang, pos, w,
                                                 static_cast<const double2*>(Jz),
                                                 static_cast<const double2*>(Ez), k, angles,
                                                 eta0, static_cast<double2*>(out));
  else
    ntff2d_kernel<float, D><<<grid, NT, 0, s>>>(n_pts, n_ang, pos, w,
                                                static_cast<const float2*>(Jz),
                                                static_cast<const float2*>(Ez), k, angles, eta0,
                                                static_cast<float2*>(out));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_ntff2d_project_grad(int32_t n_freq, int32_t n_pts, int32_t n_ang,
                                       int32_t c128, const double* pos, const double* w,
                                       const double* k, const double* angles, double eta0,
                                       const void* g_out, void* g_Jz, void* g_Ez, void* stream) {
  if (n_freq < 0 || n_pts < 0 || n_ang < 0) GDN_BAD_ARG("negative size");
  if (n_freq == 0 || n_pts == 0) return GDN_OK;
  if (!pos || !w || !k || !angles || !g_out || !g_Jz || !g_Ez) GDN_BAD_ARG("null pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid(unsigned(gdn::div_up(n_pts, NT)), n_freq);
  if (c128)
    ntff2d_grad_kernel<double><<<grid, NT, 0, s>>>(n_pts, n_ang, pos, w, k, angles, eta0,
                                                   static_cast<const double2*>(g_out),
                                                   static_cast<double2*>(g_Jz),
                                                   static_cast<double2*>(g_Ez));
  else
    ntff2d_grad_kernel<float><<<grid, NT, 0, s>>>(n_pts, n_ang, pos, w, k, angles, eta0,
                                                  static_cast<const float2*>(g_out),
                                                  static_cast<float2*>(g_Jz),
                                                  static_cast<float2*>(g_Ez));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}
