// Objective reductions on DFT phasors and the frequency-domain adjoint
// design contraction for the 2D TM path.
//
//   gdn_poynting_box_2d        monitors.py:20-70 (closed dual-grid contour flux)
//   gdn_poynting_box_2d_grad   its exact cotangent, scattered onto the phasors
//   gdn_tm_adjoint_contract    freq_adjoint.py:454-493 with _dcoef_closed :186-206
//
// The flux is a small reduction (O(n_freq x perimeter)): one CTA per
// frequency, per-thread partial sums in double, warp-shuffle then shared
// memory reduction; no atomics, so the result is deterministic.
#include "common.cuh"

namespace gdn {
namespace adj2d {

template <typename C>
__device__ __forceinline__ double re_mul_conj(C a, C b) {  // Re(a conj(b))
  return double(a.x) * double(b.x) + double(a.y) * double(b.y);
}

template <typename C>
__device__ __forceinline__ C avg(C a, C b) {
  C r;
  r.x = (a.x + b.x) * decltype(a.x)(0.5);
  r.y = (a.y + b.y) * decltype(a.x)(0.5);
  return r;
}

// Face geometry of the contour (monitors.py:52-70): the right/left faces run
// over j in (jb, jt], the top/bottom faces over i in (il, ir].
struct Box {
  int il, ir, jb, jt;
  int nx, ny;
};

template <typename C>
__global__ void poynting_kernel(Box b, double dx, double dy, const C* ez, const C* hx,
                                const C* hy, double* out) {
  const int k = blockIdx.x;
  const long long pe = (long long)b.nx * b.ny, px = (long long)b.nx * (b.ny - 1),
                  py = (long long)(b.nx - 1) * b.ny;
  const C* e = ez + k * pe;
  const C* x = hx + k * px;
  const C* y = hy + k * py;
  double acc = 0.0;
  const int nj = b.jt - b.jb, ni = b.ir - b.il;
  for (int t = threadIdx.x; t < nj; t += blockDim.x) {
    const int j = b.jb + 1 + t;
    // right face, outward +x: Sx = -1/2 Re(Ez Hy*)
    C er = avg(e[(long long)b.ir * b.ny + j], e[(long long)(b.ir + 1) * b.ny + j]);
    acc += -0.5 * re_mul_conj(er, y[(long long)b.ir * b.ny + j]) * dy;
    // left face, outward -x
    C el = avg(e[(long long)b.il * b.ny + j], e[(long long)(b.il + 1) * b.ny + j]);
    acc += 0.5 * re_mul_conj(el, y[(long long)b.il * b.ny + j]) * dy;
  }
  for (int t = threadIdx.x; t < ni; t += blockDim.x) {
    const int i = b.il + 1 + t;
    // top face, outward +y: Sy = +1/2 Re(Ez Hx*)
    C et = avg(e[(long long)i * b.ny + b.jt], e[(long long)i * b.ny + b.jt + 1]);
    acc += 0.5 * re_mul_conj(et, x[(long long)i * (b.ny - 1) + b.jt]) * dx;
    // bottom face, outward -y
    C eb = avg(e[(long long)i * b.ny + b.jb], e[(long long)i * b.ny + b.jb + 1]);
    acc += -0.5 * re_mul_conj(eb, x[(long long)i * (b.ny - 1) + b.jb]) * dx;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ double part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    acc = threadIdx.x < nw ? part[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) out[k] = acc;
  }
}

// d/d(conj z) in torch's convention of s Re(a conj(h)) is s h for a and s a for h.
template <typename C>
__device__ __forceinline__ void add_scaled(C* p, C v, double s) {
  C r = *p;
  r.x += decltype(r.x)(s * double(v.x));
  r.y += decltype(r.y)(s * double(v.y));
  *p = r;
}

template <typename C>
__global__ void poynting_grad_kernel(Box b, double dx, double dy, const C* ez, const C* hx,
                                     const C* hy, const double* g_out, C* gez, C* ghx, C* ghy) {
  const int k = blockIdx.x;
  const long long pe = (long long)b.nx * b.ny, px = (long long)b.nx * (b.ny - 1),
                  py = (long long)(b.nx - 1) * b.ny;
  const C* e = ez + k * pe;
  const C* x = hx + k * px;
  const C* y = hy + k * py;
  C* ge = gez + k * pe;
  C* gx = ghx + k * px;
  C* gy = ghy + k * py;
  const double g = g_out[k];
  const int nj = b.jt - b.jb, ni = b.ir - b.il;
  // Faces in a fixed order with a barrier between them: corner cells shared
  // by two faces are updated by one thread at a time.
  for (int face = 0; face < 4; ++face) {
    const int len = face < 2 ? nj : ni;
    for (int t = threadIdx.x; t < len; t += blockDim.x) {
      long long e0, e1, h;
      C* gh;
      const C* hv;
      double s;
      if (face < 2) {
        const int j = b.jb + 1 + t, i = face == 0 ? b.ir : b.il;
        e0 = (long long)i * b.ny + j;
        e1 = (long long)(i + 1) * b.ny + j;
        h = (long long)i * b.ny + j;
        gh = gy;
        hv = y;
        s = (face == 0 ? -0.5 : 0.5) * dy * g;
      } else {
        const int i = b.il + 1 + t, j = face == 2 ? b.jt : b.jb;
        e0 = (long long)i * b.ny + j;
        e1 = (long long)i * b.ny + j + 1;
        h = (long long)i * (b.ny - 1) + j;
        gh = gx;
        hv = x;
        s = (face == 2 ? 0.5 : -0.5) * dx * g;
      }
      const C ea = avg(e[e0], e[e1]);
      const C hh = hv[h];
      add_scaled(ge + e0, hh, 0.5 * s);
      add_scaled(ge + e1, hh, 0.5 * s);
      add_scaled(gh + h, ea, s);
    }
    __syncthreads();
  }
}

// freq_adjoint.py:454-493 for one design cell, all frequencies.
__global__ void contract_kernel(int n_cells, int K, double dt, double k_norm,
                                const double2* e_fwd, const double2* lam, const double* eps_r,
                                const double* sigma, const double2* z, double* g_sig,
                                double* g_eps, int flags) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cells) return;
  const double EPS0 = 1.0 / (1.25663706212e-06 * 299792458.0 * 299792458.0);
  const double er = eps_r[c];
  const double eps = EPS0 * er, sig = sigma[c];
  const double h = sig * dt / (2.0 * eps);
  const double ca = (1.0 - h) / (1.0 + h);
  const double cb = (dt / eps) / (1.0 + h);
  const double den = (1.0 + h) * (1.0 + h);
  const double dca_s = (-dt / eps) / den;
  const double dcb_s = (-(dt / eps) * (dt / (2.0 * eps))) / den;
  const double dca_e = EPS0 * ((sig * dt / (eps * eps)) / den);
  const double dcb_e = EPS0 * ((-(dt / (eps * eps))) / den);
  double gs = 0.0, ge = 0.0;
  for (int k = 0; k < K; ++k) {
    const double2 e = e_fwd[(long long)k * n_cells + c];
    const double2 l = lam[(long long)k * n_cells + c];
    const double2 zk = z[k];
    // en = e / z
    const double zz = zk.x * zk.x + zk.y * zk.y;
    const double2 en = make_double2((e.x * zk.x + e.y * zk.y) / zz, (e.y * zk.x - e.x * zk.y) / zz);
    const double2 cu = make_double2((e.x - ca * en.x) / cb, (e.y - ca * en.y) / cb);
    // Re(conj(l) conj(g)) = l.x g.x - l.y g.y
    const double2 g1 = make_double2(dca_s * en.x + dcb_s * cu.x, dca_s * en.y + dcb_s * cu.y);
    const double2 g2 = make_double2(dca_e * en.x + dcb_e * cu.x, dca_e * en.y + dcb_e * cu.y);
    gs += k_norm * (l.x * g1.x - l.y * g1.y);
    ge += k_norm * (l.x * g2.x - l.y * g2.y);
  }
  // The adjoint Ez phasor is recorded on the vacuum source basis; the cell's
  // own update uses c_b = (dt / eps) / (1 + h), so the adjoint amplitude
  // carries 1 / (eps_r (1 + h)) relative to vacuum. The reference undoes
  // only the eps_r part (freq_adjoint.py:474-486), which is exact for
  // h << 1 only; GDN_CONTRACT_EXACT_LOSS undoes both.
  const double scale = (flags & GDN_CONTRACT_EXACT_LOSS) ? er * (1.0 + h) : er;
  if (g_sig) g_sig[c] = scale * gs;
  if (g_eps) g_eps[c] = scale * ge;
}

static int check_box(int nx, int ny, int n_freq, const int32_t* box) {
  if (!box) GDN_BAD_ARG("box is null");
  if (n_freq < 0) GDN_BAD_ARG("n_freq < 0");
  const int il = box[0], ir = box[1], jb = box[2], jt = box[3];
  if (!(0 <= il && il < ir && ir < nx - 1 && 0 <= jb && jb < jt && jt < ny - 1))
    GDN_BAD_ARG("box (%d, %d, %d, %d) is not a valid contour on a %dx%d grid", il, ir, jb, jt,
                nx, ny);
  return GDN_OK;
}

}  // namespace adj2d
}  // namespace gdn

using namespace gdn::adj2d;

extern "C" int gdn_poynting_box_2d(int32_t nx, int32_t ny, int32_t n_freq, const int32_t box[4],
                                   double dx, double dy, int32_t c128, const void* dft_ez,
                                   const void* dft_hx, const void* dft_hy, double* out,
                                   void* stream) {
  int st = check_box(nx, ny, n_freq, box);
  if (st) return st;
  if (n_freq == 0) return GDN_OK;
  if (!dft_ez || !dft_hx || !dft_hy || !out) GDN_BAD_ARG("null phasor or output pointer");
  Box b{box[0], box[1], box[2], box[3], nx, ny};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (c128)
    poynting_kernel<double2><<<n_freq, 256, 0, s>>>(b, dx, dy, static_cast<const double2*>(dft_ez),
                                                    static_cast<const double2*>(dft_hx),
                                                    static_cast<const double2*>(dft_hy), out);
  else
    poynting_kernel<float2><<<n_freq, 256, 0, s>>>(b, dx, dy, static_cast<const float2*>(dft_ez),
                                                   static_cast<const float2*>(dft_hx),
                                                   static_cast<const float2*>(dft_hy), out);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_poynting_box_2d_grad(int32_t nx, int32_t ny, int32_t n_freq,
                                        const int32_t box[4], double dx, double dy, int32_t c128,
                                        const void* dft_ez, const void* dft_hx, const void* dft_hy,
                                        const double* g_out, void* g_ez, void* g_hx, void* g_hy,
                                        void* stream) {
  int st = check_box(nx, ny, n_freq, box);
  if (st) return st;
  if (n_freq == 0) return GDN_OK;
  if (!dft_ez || !dft_hx || !dft_hy || !g_out || !g_ez || !g_hx || !g_hy)
    GDN_BAD_ARG("null pointer");
  Box b{box[0], box[1], box[2], box[3], nx, ny};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (c128)
    poynting_grad_kernel<double2><<<n_freq, 256, 0, s>>>(
        b, dx, dy, static_cast<const double2*>(dft_ez), static_cast<const double2*>(dft_hx),
        static_cast<const double2*>(dft_hy), g_out, static_cast<double2*>(g_ez),
        static_cast<double2*>(g_hx), static_cast<double2*>(g_hy));
  else
    poynting_grad_kernel<float2><<<n_freq, 256, 0, s>>>(
        b, dx, dy, static_cast<const float2*>(dft_ez), static_cast<const float2*>(dft_hx),
        static_cast<const float2*>(dft_hy), g_out, static_cast<float2*>(g_ez),
        static_cast<float2*>(g_hx), static_cast<float2*>(g_hy));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_tm_adjoint_contract(int32_t n_cells, int32_t n_freq, double dt, double k_norm,
                                       const void* e_fwd, const void* lam, const double* eps_r,
                                       const double* sigma, const void* z, double* grad_sigma,
                                       double* grad_eps_r, int32_t flags, void* stream) {
  if (n_cells < 0 || n_freq < 0) GDN_BAD_ARG("negative size");
  if (n_cells == 0) return GDN_OK;
  if (!e_fwd || !lam || !eps_r || !sigma || !z) GDN_BAD_ARG("null input pointer");
  if (!grad_sigma && !grad_eps_r) GDN_BAD_ARG("both gradient outputs are null");
  contract_kernel<<<unsigned(gdn::div_up(n_cells, 256)), 256, 0,
                    static_cast<cudaStream_t>(stream)>>>(
      n_cells, n_freq, dt, k_norm, static_cast<const double2*>(e_fwd),
      static_cast<const double2*>(lam), eps_r, sigma, static_cast<const double2*>(z), grad_sigma,
      grad_eps_r, flags);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}
