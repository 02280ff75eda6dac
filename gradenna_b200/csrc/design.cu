// The topology-optimisation design transform (topopt.py:55-127 of the
// reference): rho = tanh_projection(conic_filter(sigmoid(theta), R), beta,
// eta) for a batch of B designs of H x W cells, and its exact backward.
//
// conic_filter is the boundary-renormalised correlation
//   f(p) = sum_o w_o s(p + o) / sum_o w_o [p + o inside],
//   w_o = max(0, 1 - |o| / R),  |o_x|, |o_y| <= n = ceil(R) - 1,
// (the kernel is symmetric, so correlation and convolution coincide), and
// tanh_projection(f) = (tanh(beta eta) + tanh(beta (f - eta))) /
//                      (tanh(beta eta) + tanh(beta (1 - eta))).
// One thread per output cell; the (2n+1)^2 weights sit in shared memory and
// the sigmoid of each neighbour is evaluated on the fly (the designs are a
// few hundred cells a side, so re-reading theta from L1/L2 is cheap).
//
// Backward: with g = dL/drho, gf = g * beta sech^2(beta (f - eta)) / D,
// dL/ds(q) = sum_o w_o gf(q - o) / den(q - o), dL/dtheta = dL/ds * s (1 - s);
// the forward stores f and the window norm den for it.
// No reference counterpart as CUDA: the reference evaluates the transform
// with jax (fftconvolve) and differentiates it with jax.grad.
#include "common.cuh"

namespace gdn {
namespace design {

constexpr int MAXN = 24;  // half width of the filter window (R <= 25 cells)

__device__ __forceinline__ double sigm(double x) { return 1.0 / (1.0 + exp(-x)); }

__global__ void design_fwd(const double* __restrict__ theta, int B, int H, int W,
                           const double* __restrict__ kern, int n, double beta, double eta,
                           double* __restrict__ filt, double* __restrict__ norm,
                           double* __restrict__ rho) {
  extern __shared__ double sw[];
  const int k = 2 * n + 1;
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) sw[q] = kern[q];
  __syncthreads();
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (long long)B * H * W) return;
  const int b = int(c / ((long long)H * W));
  const int rem = int(c - (long long)b * H * W);
  const int i = rem / W, j = rem - (rem / W) * W;
  const double* th = theta + (long long)b * H * W;
  double num = 0.0, den = 0.0;
  for (int a = -n; a <= n; ++a) {
    if (i + a < 0 || i + a >= H) continue;
    for (int d = -n; d <= n; ++d) {
      if (j + d < 0 || j + d >= W) continue;
      const double wt = sw[(a + n) * k + (d + n)];
      num += wt * sigm(th[(i + a) * W + (j + d)]);
      den += wt;
    }
  }
  const double f = num / den;
  filt[c] = f;
  norm[c] = den;
  const double te = tanh(beta * eta);
  rho[c] = (te + tanh(beta * (f - eta))) / (te + tanh(beta * (1.0 - eta)));
}

__global__ void design_bwd(const double* __restrict__ theta, const double* __restrict__ filt,
                           const double* __restrict__ norm, const double* __restrict__ g_rho,
                           int B, int H, int W,
                           const double* __restrict__ kern, int n, double beta, double eta,
                           double* __restrict__ g_theta) {
  extern __shared__ double sw[];
  const int k = 2 * n + 1;
  for (int q = threadIdx.x; q < k * k; q += blockDim.x) sw[q] = kern[q];
  __syncthreads();
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (long long)B * H * W) return;
  const int b = int(c / ((long long)H * W));
  const int rem = int(c - (long long)b * H * W);
  const int i = rem / W, j = rem - (rem / W) * W;
  const long long base = (long long)b * H * W;
  const double D = tanh(beta * eta) + tanh(beta * (1.0 - eta));
  double gs = 0.0;
  for (int a = -n; a <= n; ++a) {
    const int pi = i - a;
    if (pi < 0 || pi >= H) continue;
    for (int d = -n; d <= n; ++d) {
      const int pj = j - d;
      if (pj < 0 || pj >= W) continue;
      const long long p = base + pi * W + pj;
      const double t = tanh(beta * (filt[p] - eta));
      const double gf = g_rho[p] * beta * (1.0 - t * t) / D;
      gs += sw[(a + n) * k + (d + n)] * gf / norm[p];
    }
  }
  const double s = sigm(theta[c]);
  g_theta[c] = gs * s * (1.0 - s);
}

}  // namespace design
}  // namespace gdn

using namespace gdn::design;

extern "C" int gdn_design_forward(const double* theta, int32_t B, int32_t H, int32_t W,
                                  const double* kern, int32_t n, double beta, double eta,
                                  double* filt, double* norm, double* rho, void* stream) {
  if (!theta || !kern || !filt || !norm || !rho || B <= 0 || H <= 0 || W <= 0)
    GDN_BAD_ARG("invalid arguments");
  if (n < 0 || n > MAXN) GDN_BAD_ARG("filter half width %d outside [0, %d]", n, MAXN);
  const long long cells = (long long)B * H * W;
  const int k = 2 * n + 1;
  design_fwd<<<unsigned((cells + 255) / 256), 256, sizeof(double) * k * k,
               static_cast<cudaStream_t>(stream)>>>(theta, B, H, W, kern, n, beta, eta, filt, norm,
                                                    rho);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_design_backward(const double* theta, const double* filt, const double* norm,
                                   const double* g_rho, int32_t B, int32_t H, int32_t W,
                                   const double* kern, int32_t n, double beta, double eta,
                                   double* g_theta, void* stream) {
  if (!theta || !filt || !norm || !g_rho || !kern || !g_theta || B <= 0 || H <= 0 || W <= 0)
    GDN_BAD_ARG("invalid arguments");
  if (n < 0 || n > MAXN) GDN_BAD_ARG("filter half width %d outside [0, %d]", n, MAXN);
  const long long cells = (long long)B * H * W;
  const int k = 2 * n + 1;
  design_bwd<<<unsigned((cells + 255) / 256), 256, sizeof(double) * k * k,
               static_cast<cudaStream_t>(stream)>>>(theta, filt, norm, g_rho, B, H, W, kern, n,
                                                    beta, eta, g_theta);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}
