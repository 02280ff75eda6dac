// Kernels of the design surrogate (a 2D U-Net over design densities): BF16
// tensor-core convolutions with FP32 accumulation and their weight
// gradients, 2x2 max pooling, nearest x2 upsampling, the output head's loss
// gradient and Adam.
//
// Layout: activations are NHWC bfloat16. A tensor may be a channel slice
// [c0, c0 + C) of a wider buffer (row stride = the buffer's channels), so the
// U-Net's skip concatenations are written in place by their producers.
// Weights are [K][Cout] bfloat16 with K = taps * Cin, k = tap * Cin + ci and
// tap = (dy + 1) * 3 + (dx + 1) for 3x3 kernels (taps = 9), tap 0 for 1x1.
//
// Convolution = implicit GEMM (rows = pixels, columns = output channels,
// reduction over (tap, input channel)). A CTA of four warps computes a
// 64 x 64 tile as 2 x 2 warp tiles of 32 x 32 (2 x 2 bf16 16x16x16 MMA
// fragments each); the reduction runs in 32-wide steps whose activation
// (im2col rows gathered with zero padding at the image border) and weight
// tiles are staged in shared memory by 16-byte cp.async copies, double
// buffered so the next step's loads overlap this step's MMAs. Layers whose
// channel counts are not multiples of 8 (the 1-channel density input and the
// 3-channel head) take a scalar staging path.
//
// Activations are leaky ReLUs, y = x > 0 ? x : slope * x (slope 0 = ReLU).
// The input gradient of a convolution is the same kernel run on the output
// gradient with point-reflected, transposed weights (flip_weights). Its
// epilogue can multiply by (x > 0 ? 1 : slope) for the forward input x of
// the layer: in this network every convolution input is an activation output
// or a max-pool, upsampling or concatenation of activation outputs, whose
// sign is the sign of the producing pre-activation, so that factor is
// exactly the activation derivative of the producing layers.
#include <mma.h>

#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"

namespace gdn {
namespace surr {

using namespace nvcuda;
using bf16 = __nv_bfloat16;

constexpr int BM = 64, BN = 64, BK = 32, THREADS = 128;
constexpr int LDA = BK + 8;  // bf16 elements per staged activation row
constexpr int LDB = BN + 8;  // bf16 elements per staged weight / gradient row
constexpr int LDT = BM + 8;  // bf16 elements per staged im2col^T row (weight gradient)
constexpr int LDC = BN + 4;  // floats per accumulator row

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int n = valid ? 16 : 0;  // 0 source bytes = zero fill
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

struct ConvArgs {
  const bf16* in;
  int in_stride, in_c0;
  int N, H, W, Cin, taps;
  const bf16* w;
  const float* bias;
  int Cout, relu;
  float slope;
  bf16* out;
  int out_stride, out_c0;
  float* out32;
  const bf16* mask;
  int mask_stride, mask_c0;
};

struct PixelPos {
  int n, y, x;
  bool ok;
};

__device__ __forceinline__ PixelPos pixel_pos(long long p, long long P, int H, int W) {
  PixelPos r;
  r.ok = p < P;
  const long long hw = (long long)H * W;
  const long long pp = r.ok ? p : 0;
  r.n = int(pp / hw);
  const int rem = int(pp - (long long)r.n * hw);
  r.y = rem / W;
  r.x = rem - r.y * W;
  return r;
}

// out = act(bias + conv(in, w)) on a 64-pixel x 64-channel tile.
// VA: Cin % 32 == 0 and 16-byte aligned activation rows (vector staging of
// the im2col tile); VB: Cout % 8 == 0 (vector staging of the weight tile).
template <bool VA, bool VB>
__global__ void __launch_bounds__(THREADS) conv_fwd(ConvArgs a) {
  struct Stage {
    bf16 A[2][BM][LDA];
    bf16 B[2][BK][LDB];
  };
  __shared__ __align__(128) unsigned char raw[sizeof(Stage) > sizeof(float) * BM * LDC
                                                  ? sizeof(Stage)
                                                  : sizeof(float) * BM * LDC];
  Stage& st = *reinterpret_cast<Stage*>(raw);
  float(*sC)[LDC] = reinterpret_cast<float(*)[LDC]>(raw);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const long long P = (long long)a.N * a.H * a.W;
  const long long p0 = (long long)blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int K = a.taps * a.Cin;
  const int nk = (K + BK - 1) / BK;

  // Vector staging: thread t copies 8 channels (chunk t % 4) of rows t / 4
  // and t / 4 + 32 of the im2col tile.
  const int chunkA = tid & 3;
  PixelPos rowpos[2];
  if (VA) {
    rowpos[0] = pixel_pos(p0 + (tid >> 2), P, a.H, a.W);
    rowpos[1] = pixel_pos(p0 + (tid >> 2) + 32, P, a.H, a.W);
  }

  auto load_stage = [&](int s, int k0) {
    if (VA) {
      const int tap = k0 / a.Cin, ci0 = k0 - tap * a.Cin;
      const int dy = a.taps == 9 ? tap / 3 - 1 : 0, dx = a.taps == 9 ? tap % 3 - 1 : 0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const PixelPos& q = rowpos[h];
        const int y = q.y + dy, x = q.x + dx;
        const bool ok = q.ok && y >= 0 && y < a.H && x >= 0 && x < a.W;
        const bf16* src = ok ? a.in + (((long long)q.n * a.H + y) * a.W + x) * a.in_stride +
                                   a.in_c0 + ci0 + chunkA * 8
                             : a.in;
        cp_async16(&st.A[s][(tid >> 2) + 32 * h][chunkA * 8], src, ok);
      }
    } else {
      for (int q = tid; q < BM * BK; q += THREADS) {
        const int r = q / BK, kk = q - r * BK;
        const int k = k0 + kk;
        bf16 v = __float2bfloat16(0.f);
        const PixelPos pp = pixel_pos(p0 + r, P, a.H, a.W);
        if (pp.ok && k < K) {
          const int tap = k / a.Cin, ci = k - tap * a.Cin;
          const int dy = a.taps == 9 ? tap / 3 - 1 : 0, dx = a.taps == 9 ? tap % 3 - 1 : 0;
          const int y = pp.y + dy, x = pp.x + dx;
          if (y >= 0 && y < a.H && x >= 0 && x < a.W)
            v = a.in[(((long long)pp.n * a.H + y) * a.W + x) * a.in_stride + a.in_c0 + ci];
        }
        st.A[s][r][kk] = v;
      }
    }
    if (VB) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int v = tid + THREADS * h;
        const int r = v >> 3, ch = v & 7;
        const int k = k0 + r, co = n0 + ch * 8;
        const bool ok = k < K && co < a.Cout;
        cp_async16(&st.B[s][r][ch * 8], ok ? a.w + (long long)k * a.Cout + co : a.w, ok);
      }
    } else {
      for (int q = tid; q < BK * BN; q += THREADS) {
        const int r = q / BN, c = q - r * BN;
        const int k = k0 + r, co = n0 + c;
        st.B[s][r][c] = (k < K && co < a.Cout) ? a.w[(long long)k * a.Cout + co]
                                               : __float2bfloat16(0.f);
      }
    }
    cp_async_commit();
  };

  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.0f);

  load_stage(0, 0);
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    if (kt + 1 < nk) {
      load_stage(s ^ 1, (kt + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < BK; ks += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> fa[2];
      wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) wmma::load_matrix_sync(fa[i], &st.A[s][wm * 32 + i * 16][ks], LDA);
#pragma unroll
      for (int j = 0; j < 2; ++j) wmma::load_matrix_sync(fb[j], &st.B[s][ks][wn * 32 + j * 16], LDB);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
      wmma::store_matrix_sync(&sC[wm * 32 + i * 16][wn * 32 + j * 16], acc[i][j], LDC,
                              wmma::mem_row_major);
  __syncthreads();
  for (int q = tid; q < BM * BN; q += THREADS) {
    const int r = q / BN, c = q - r * BN;
    const long long p = p0 + r;
    const int co = n0 + c;
    if (p >= P || co >= a.Cout) continue;
    float v = sC[r][c] + (a.bias ? a.bias[co] : 0.f);
    if (a.relu && !(v > 0.f)) v *= a.slope;
    if (a.mask && !(__bfloat162float(a.mask[p * a.mask_stride + a.mask_c0 + co]) > 0.f)) v *= a.slope;
    if (a.out) a.out[p * a.out_stride + a.out_c0 + co] = __float2bfloat16(v);
    if (a.out32) a.out32[p * a.Cout + co] = v;
  }
}

struct WgradArgs {
  const bf16* in;
  int in_stride, in_c0;
  int N, H, W, Cin, taps;
  const bf16* g;
  int g_stride, g_c0;
  int Cout;
  float* dw;
  float* db;
  int pix_per_split;
};

// dw[k][co] += sum_p im2col(in)[p][k] * g[p][co] over this CTA's slice of
// pixels (split-K over blockIdx.z, FP32 atomics); db[co] += sum_p g[p][co].
// V: Cin, Cout, strides and offsets multiples of 8 (vector staging).
template <bool V>
__global__ void __launch_bounds__(THREADS) conv_wgrad(WgradArgs a) {
  struct Stage {
    bf16 T[2][BK][LDT];  // im2col^T: [pixel][k]
    bf16 G[2][BK][LDB];  // [pixel][co]
  };
  __shared__ __align__(128) unsigned char raw[sizeof(Stage) > sizeof(float) * BM * LDC
                                                  ? sizeof(Stage)
                                                  : sizeof(float) * BM * LDC];
  Stage& st = *reinterpret_cast<Stage*>(raw);
  float(*sC)[LDC] = reinterpret_cast<float(*)[LDC]>(raw);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const long long P = (long long)a.N * a.H * a.W;
  const int K = a.taps * a.Cin;
  const int k0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const long long pb = (long long)blockIdx.z * a.pix_per_split;
  const long long pe = min(P, pb + a.pix_per_split);
  const int nsteps = int((pe - pb + BK - 1) / BK);

  // Vector staging: thread t copies chunk t % 8 (8 reduction indices) of
  // pixel rows t / 8 and t / 8 + 16; the chunk's tap is fixed per thread.
  const int chunk = tid & 7;
  const int kq = k0 + chunk * 8;
  const bool kval = kq < K;
  const int tapq = kval ? kq / a.Cin : 0;
  const int ciq = kq - tapq * a.Cin;
  const int dyq = a.taps == 9 ? tapq / 3 - 1 : 0, dxq = a.taps == 9 ? tapq % 3 - 1 : 0;

  auto load_stage = [&](int s, long long q0) {
    if (V) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = (tid >> 3) + 16 * h;
        const PixelPos pp = pixel_pos(q0 + r, pe, a.H, a.W);
        const int y = pp.y + dyq, x = pp.x + dxq;
        const bool ok = kval && pp.ok && y >= 0 && y < a.H && x >= 0 && x < a.W;
        const bf16* src =
            ok ? a.in + (((long long)pp.n * a.H + y) * a.W + x) * a.in_stride + a.in_c0 + ciq : a.in;
        cp_async16(&st.T[s][r][chunk * 8], src, ok);
        const int co = n0 + chunk * 8;
        const bool okg = pp.ok && co < a.Cout;
        cp_async16(&st.G[s][r][chunk * 8],
                   okg ? a.g + (q0 + r) * a.g_stride + a.g_c0 + co : a.g, okg);
      }
    } else {
      for (int q = tid; q < BK * BM; q += THREADS) {
        const int r = q / BM, kk = q - r * BM;
        const int k = k0 + kk;
        bf16 v = __float2bfloat16(0.f);
        const PixelPos pp = pixel_pos(q0 + r, pe, a.H, a.W);
        if (pp.ok && k < K) {
          const int tap = k / a.Cin, ci = k - tap * a.Cin;
          const int dy = a.taps == 9 ? tap / 3 - 1 : 0, dx = a.taps == 9 ? tap % 3 - 1 : 0;
          const int y = pp.y + dy, x = pp.x + dx;
          if (y >= 0 && y < a.H && x >= 0 && x < a.W)
            v = a.in[(((long long)pp.n * a.H + y) * a.W + x) * a.in_stride + a.in_c0 + ci];
        }
        st.T[s][r][kk] = v;
      }
      for (int q = tid; q < BK * BN; q += THREADS) {
        const int r = q / BN, c = q - r * BN;
        const long long p = q0 + r;
        const int co = n0 + c;
        st.G[s][r][c] = (p < pe && co < a.Cout) ? a.g[p * a.g_stride + a.g_c0 + co]
                                                : __float2bfloat16(0.f);
      }
    }
    cp_async_commit();
  };

  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) wmma::fill_fragment(acc[i][j], 0.0f);
  float bsum = 0.f;
  const bool do_bias = a.db && blockIdx.x == 0 && tid < BN;

  if (nsteps > 0) load_stage(0, pb);
  for (int t = 0; t < nsteps; ++t) {
    const int s = t & 1;
    if (t + 1 < nsteps) {
      load_stage(s ^ 1, pb + (long long)(t + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (do_bias)
      for (int r = 0; r < BK; ++r) bsum += __bfloat162float(st.G[s][r][tid]);
#pragma unroll
    for (int ks = 0; ks < BK; ks += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::col_major> fa[2];
      wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> fb[2];
#pragma unroll
      for (int i = 0; i < 2; ++i) wmma::load_matrix_sync(fa[i], &st.T[s][ks][wm * 32 + i * 16], LDT);
#pragma unroll
      for (int j = 0; j < 2; ++j) wmma::load_matrix_sync(fb[j], &st.G[s][ks][wn * 32 + j * 16], LDB);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], fa[i], fb[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
      wmma::store_matrix_sync(&sC[wm * 32 + i * 16][wn * 32 + j * 16], acc[i][j], LDC,
                              wmma::mem_row_major);
  __syncthreads();
  for (int q = tid; q < BM * BN; q += THREADS) {
    const int r = q / BN, c = q - r * BN;
    const int k = k0 + r, co = n0 + c;
    if (k < K && co < a.Cout) atomicAdd(&a.dw[(long long)k * a.Cout + co], sC[r][c]);
  }
  if (do_bias && n0 + tid < a.Cout) atomicAdd(&a.db[n0 + tid], bsum);
}

// Weights of the input-gradient convolution: wt[tf * Cout + co][ci] =
// w[tap * Cin + ci][co] with tf = taps - 1 - tap the point-reflected tap.
__global__ void flip_weights(const bf16* __restrict__ w, int Cin, int Cout, int taps,
                             bf16* __restrict__ wt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)taps * Cin * Cout;
  if (i >= total) return;
  const int co = int(i % Cout);
  const long long kc = i / Cout;
  const int ci = int(kc % Cin), tap = int(kc / Cin);
  const int tf = taps - 1 - tap;
  wt[((long long)tf * Cout + co) * Cin + ci] = w[i];
}

// 2x2 max pooling (H, W even) keeping the winning position (0..3, row major
// within the window; the first maximum wins) for the backward pass.
__global__ void maxpool2_fwd(const bf16* __restrict__ in, int in_stride, int in_c0, int N, int H,
                             int W, int C, bf16* __restrict__ out, unsigned char* __restrict__ arg) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Ho = H / 2, Wo = W / 2;
  if (i >= (long long)N * Ho * Wo * C) return;
  const int c = int(i % C);
  const long long po = i / C;
  const int n = int(po / ((long long)Ho * Wo));
  const int rem = int(po - (long long)n * Ho * Wo);
  const int yo = rem / Wo, xo = rem - (rem / Wo) * Wo;
  float best = -INFINITY;
  int bi = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int y = 2 * yo + (q >> 1), x = 2 * xo + (q & 1);
    const float v = __bfloat162float(in[(((long long)n * H + y) * W + x) * in_stride + in_c0 + c]);
    if (v > best) {
      best = v;
      bi = q;
    }
  }
  out[i] = __float2bfloat16(best);
  arg[i] = (unsigned char)bi;
}

// gin[window winner] += gout (the other three positions are unchanged).
__global__ void maxpool2_bwd_acc(const bf16* __restrict__ gout, const unsigned char* __restrict__ arg,
                                 int N, int H, int W, int C, bf16* __restrict__ gin,
                                 int gin_stride, int gin_c0) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Ho = H / 2, Wo = W / 2;
  if (i >= (long long)N * Ho * Wo * C) return;
  const int c = int(i % C);
  const long long po = i / C;
  const int n = int(po / ((long long)Ho * Wo));
  const int rem = int(po - (long long)n * Ho * Wo);
  const int yo = rem / Wo, xo = rem - (rem / Wo) * Wo;
  const int q = arg[i];
  const int y = 2 * yo + (q >> 1), x = 2 * xo + (q & 1);
  bf16* dst = gin + (((long long)n * H + y) * W + x) * gin_stride + gin_c0 + c;
  *dst = __float2bfloat16(__bfloat162float(*dst) + __bfloat162float(gout[i]));
}

// Nearest-neighbour x2 upsampling into a channel slice, and its gradient.
__global__ void upsample2_fwd(const bf16* __restrict__ in, int N, int H, int W, int C,
                              bf16* __restrict__ out, int out_stride, int out_c0) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int Ho = 2 * H, Wo = 2 * W;
  if (i >= (long long)N * Ho * Wo * C) return;
  const int c = int(i % C);
  const long long po = i / C;
  const int n = int(po / ((long long)Ho * Wo));
  const int rem = int(po - (long long)n * Ho * Wo);
  const int y = rem / Wo, x = rem - (rem / Wo) * Wo;
  out[po * out_stride + out_c0 + c] = in[(((long long)n * H + y / 2) * W + x / 2) * C + c];
}

__global__ void upsample2_bwd(const bf16* __restrict__ gout, int g_stride, int g_c0, int N, int H,
                              int W, int C, bf16* __restrict__ gin) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)N * H * W * C) return;
  const int c = int(i % C);
  const long long p = i / C;
  const int n = int(p / ((long long)H * W));
  const int rem = int(p - (long long)n * H * W);
  const int y = rem / W, x = rem - (rem / W) * W;
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const long long po = ((long long)n * 2 * H + 2 * y + (q >> 1)) * (2 * W) + 2 * x + (q & 1);
    s += __bfloat162float(gout[po * g_stride + g_c0 + c]);
  }
  gin[i] = __float2bfloat16(s);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// mean[n] += sum_hw out32[n, hw, c] / HW (mean zeroed by the launcher).
__global__ void chan_mean(const float* __restrict__ out32, int HW, int C, int c,
                          float* __restrict__ mean) {
  const int n = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float v = i < HW ? out32[((long long)n * HW + i) * C + c] : 0.f;
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) atomicAdd(&mean[n], v / float(HW));
}

// Loss gradient of the head output out32[N, HW, C] (channels 0, 1 = field,
// channel 2 = power density whose spatial mean is the power prediction):
//   L = wf * mean_{n,hw,k<2} (out_k - tf_k)^2 + wp * mean_n (mean_hw out_2 - tp)^2
// or, without targets, the gradient of sum_n pw[n] * mean_hw out_2 (field
// channels get zero gradient). Writes the BF16 gradient and adds L to *loss.
__global__ void head_grad(const float* __restrict__ out32, long long NHW, int HW, int C,
                          const float* __restrict__ tf, const float* __restrict__ tp,
                          const float* __restrict__ pw, const float* __restrict__ mean, float wf,
                          float wp, bf16* __restrict__ grad, float* __restrict__ loss) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < NHW) {
    const int n = int(i / HW);
    const float nf = float(NHW / HW);
    for (int k = 0; k < C; ++k) {
      float gk = 0.f;
      if (k < 2) {
        if (tf) {
          const float d = out32[i * C + k] - tf[i * 2 + k];
          gk = 2.f * wf * d / float(2 * NHW);
          l += wf * d * d / float(2 * NHW);
        }
      } else if (k == 2) {
        if (tp) {
          const float e = mean[n] - tp[n];
          gk = 2.f * wp * e / (nf * float(HW));
          if (i % HW == 0) l += wp * e * e / nf;
        } else {
          gk = (pw ? pw[n] : 1.f) / float(HW);
        }
      }
      grad[i * C + k] = __float2bfloat16(gk);
    }
  }
  l = warp_sum(l);
  if (loss && (threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// Adam bias-correction factors for the next step: hyper = {step, lr, 1 - b1^t, 1 - b2^t}.
__global__ void adam_prepare(float* hyper, float b1, float b2) {
  const float t = hyper[0] + 1.f;
  hyper[0] = t;
  hyper[2] = 1.f - powf(b1, t);
  hyper[3] = 1.f - powf(b2, t);
}

// Adam on FP32 master weights with a BF16 copy for the convolutions.
__global__ void adam_step(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, bf16* __restrict__ w16, long long n,
                          const float* __restrict__ hyper, float b1, float b2, float eps) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float lr = hyper[1], c1 = hyper[2], c2 = hyper[3];
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (w16) w16[i] = __float2bfloat16(wi);
}

__global__ void f32_to_bf16(const float* __restrict__ a, bf16* __restrict__ b, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16(a[i]);
}

inline unsigned blocks_for(long long n, int t = 256) { return unsigned((n + t - 1) / t); }

inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace surr
}  // namespace gdn

using namespace gdn::surr;

#define GDN_S(x) static_cast<cudaStream_t>(x)

extern "C" int gdn_sur_conv_fwd(const void* in, int32_t in_stride, int32_t in_c0, int32_t N,
                                int32_t H, int32_t W, int32_t Cin, int32_t taps, const void* w,
                                const float* bias, int32_t Cout, int32_t relu, float slope, void* out,
                                int32_t out_stride, int32_t out_c0, float* out32, const void* mask,
                                int32_t mask_stride, int32_t mask_c0, void* stream) {
  if (N <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0 || (taps != 1 && taps != 9))
    GDN_BAD_ARG("invalid convolution shape");
  if (!in || !w || (!out && !out32)) GDN_BAD_ARG("null pointer");
  if (in_c0 < 0 || in_c0 + Cin > in_stride) GDN_BAD_ARG("input channel slice out of range");
  if (out && (out_c0 < 0 || out_c0 + Cout > out_stride)) GDN_BAD_ARG("output channel slice out of range");
  if (mask && (mask_c0 < 0 || mask_c0 + Cout > mask_stride)) GDN_BAD_ARG("mask channel slice out of range");
  ConvArgs a{static_cast<const bf16*>(in), in_stride, in_c0, N, H, W, Cin, taps,
             static_cast<const bf16*>(w), bias, Cout, relu, slope, static_cast<bf16*>(out),
             out_stride, out_c0, out32, static_cast<const bf16*>(mask), mask_stride, mask_c0};
  const long long P = (long long)N * H * W;
  const dim3 grid(unsigned((P + BM - 1) / BM), unsigned((Cout + BN - 1) / BN));
  const bool va = Cin % 32 == 0 && in_stride % 8 == 0 && in_c0 % 8 == 0 && al16(in);
  const bool vb = Cout % 8 == 0 && al16(w);
  cudaStream_t s = GDN_S(stream);
  if (va && vb)
    conv_fwd<true, true><<<grid, THREADS, 0, s>>>(a);
  else if (va)
    conv_fwd<true, false><<<grid, THREADS, 0, s>>>(a);
  else if (vb)
    conv_fwd<false, true><<<grid, THREADS, 0, s>>>(a);
  else
    conv_fwd<false, false><<<grid, THREADS, 0, s>>>(a);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_conv_wgrad(const void* in, int32_t in_stride, int32_t in_c0, int32_t N,
                                  int32_t H, int32_t W, int32_t Cin, int32_t taps, const void* g,
                                  int32_t g_stride, int32_t g_c0, int32_t Cout, float* dw, float* db,
                                  void* stream) {
  if (N <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0 || (taps != 1 && taps != 9))
    GDN_BAD_ARG("invalid convolution shape");
  if (!in || !g || !dw) GDN_BAD_ARG("null pointer");
  if (in_c0 < 0 || in_c0 + Cin > in_stride || g_c0 < 0 || g_c0 + Cout > g_stride)
    GDN_BAD_ARG("channel slice out of range");
  const long long P = (long long)N * H * W;
  const int K = taps * Cin;
  const unsigned gx = unsigned((K + BM - 1) / BM), gy = unsigned((Cout + BN - 1) / BN);
  // Split the pixel reduction so the grid holds about four CTAs per SM, with
  // at least 256 pixels per split.
  long long splits = std::max<long long>(1, (148LL * 4) / (long long)(gx * gy));
  splits = std::min<long long>(splits, std::max<long long>(1, P / 256));
  long long per = (P + splits - 1) / splits;
  per = (per + BK - 1) / BK * BK;
  splits = (P + per - 1) / per;
  WgradArgs a{static_cast<const bf16*>(in), in_stride, in_c0, N, H, W, Cin, taps,
              static_cast<const bf16*>(g), g_stride, g_c0, Cout, dw, db, int(per)};
  const bool v = Cin % 8 == 0 && Cout % 8 == 0 && in_stride % 8 == 0 && in_c0 % 8 == 0 &&
                 g_stride % 8 == 0 && g_c0 % 8 == 0 && al16(in) && al16(g);
  const dim3 grid(gx, gy, unsigned(splits));
  if (v)
    conv_wgrad<true><<<grid, THREADS, 0, GDN_S(stream)>>>(a);
  else
    conv_wgrad<false><<<grid, THREADS, 0, GDN_S(stream)>>>(a);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_flip_weights(const void* w, int32_t Cin, int32_t Cout, int32_t taps,
                                    void* wt, void* stream) {
  if (!w || !wt || Cin <= 0 || Cout <= 0 || (taps != 1 && taps != 9)) GDN_BAD_ARG("invalid arguments");
  const long long n = (long long)taps * Cin * Cout;
  flip_weights<<<blocks_for(n), 256, 0, GDN_S(stream)>>>(static_cast<const bf16*>(w), Cin, Cout,
                                                         taps, static_cast<bf16*>(wt));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_maxpool2(const void* in, int32_t in_stride, int32_t in_c0, int32_t N,
                                int32_t H, int32_t W, int32_t C, void* out, void* arg, void* stream) {
  if (!in || !out || !arg || N <= 0 || C <= 0 || H < 2 || W < 2 || (H & 1) || (W & 1))
    GDN_BAD_ARG("invalid pooling arguments");
  if (in_c0 < 0 || in_c0 + C > in_stride) GDN_BAD_ARG("channel slice out of range");
  const long long n = (long long)N * (H / 2) * (W / 2) * C;
  maxpool2_fwd<<<blocks_for(n), 256, 0, GDN_S(stream)>>>(static_cast<const bf16*>(in), in_stride,
                                                          in_c0, N, H, W, C, static_cast<bf16*>(out),
                                                          static_cast<unsigned char*>(arg));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_maxpool2_grad_acc(const void* gout, const void* arg, int32_t N, int32_t H,
                                         int32_t W, int32_t C, void* gin, int32_t gin_stride,
                                         int32_t gin_c0, void* stream) {
  if (!gout || !arg || !gin || N <= 0 || C <= 0 || H < 2 || W < 2 || (H & 1) || (W & 1))
    GDN_BAD_ARG("invalid pooling arguments");
  if (gin_c0 < 0 || gin_c0 + C > gin_stride) GDN_BAD_ARG("channel slice out of range");
  const long long n = (long long)N * (H / 2) * (W / 2) * C;
  maxpool2_bwd_acc<<<blocks_for(n), 256, 0, GDN_S(stream)>>>(
      static_cast<const bf16*>(gout), static_cast<const unsigned char*>(arg), N, H, W, C,
      static_cast<bf16*>(gin), gin_stride, gin_c0);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_upsample2(const void* in, int32_t N, int32_t H, int32_t W, int32_t C,
                                 void* out, int32_t out_stride, int32_t out_c0, void* stream) {
  if (!in || !out || N <= 0 || H <= 0 || W <= 0 || C <= 0) GDN_BAD_ARG("invalid arguments");
  if (out_c0 < 0 || out_c0 + C > out_stride) GDN_BAD_ARG("channel slice out of range");
  const long long n = (long long)N * 4 * H * W * C;
  upsample2_fwd<<<blocks_for(n), 256, 0, GDN_S(stream)>>>(static_cast<const bf16*>(in), N, H, W, C,
                                                           static_cast<bf16*>(out), out_stride, out_c0);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_upsample2_grad(const void* gout, int32_t g_stride, int32_t g_c0, int32_t N,
                                      int32_t H, int32_t W, int32_t C, void* gin, void* stream) {
  if (!gout || !gin || N <= 0 || H <= 0 || W <= 0 || C <= 0) GDN_BAD_ARG("invalid arguments");
  if (g_c0 < 0 || g_c0 + C > g_stride) GDN_BAD_ARG("channel slice out of range");
  const long long n = (long long)N * H * W * C;
  upsample2_bwd<<<blocks_for(n), 256, 0, GDN_S(stream)>>>(static_cast<const bf16*>(gout), g_stride,
                                                           g_c0, N, H, W, C, static_cast<bf16*>(gin));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_head_grad(const float* out32, int32_t N, int32_t HW, int32_t C,
                                 const float* target_field, const float* target_power,
                                 const float* power_weight, float wf, float wp, float* mean,
                                 void* grad, float* loss, void* stream) {
  if (!out32 || !mean || !grad || N <= 0 || HW <= 0 || C < 3) GDN_BAD_ARG("invalid arguments");
  cudaStream_t s = GDN_S(stream);
  GDN_TRY_CUDA(cudaMemsetAsync(mean, 0, sizeof(float) * N, s));
  chan_mean<<<dim3(blocks_for(HW), unsigned(N)), 256, 0, s>>>(out32, HW, C, 2, mean);
  const long long nhw = (long long)N * HW;
  head_grad<<<blocks_for(nhw), 256, 0, s>>>(out32, nhw, HW, C, target_field, target_power,
                                            power_weight, mean, wf, wp, static_cast<bf16*>(grad),
                                            loss);
  gdn::count_launches(2);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_adam(float* w, const float* g, float* m, float* v, void* w16, int64_t n,
                            float* hyper, float b1, float b2, float eps, void* stream) {
  if (!w || !g || !m || !v || !hyper || n < 0) GDN_BAD_ARG("invalid arguments");
  cudaStream_t s = GDN_S(stream);
  adam_prepare<<<1, 1, 0, s>>>(hyper, b1, b2);
  if (n > 0)
    adam_step<<<blocks_for(n), 256, 0, s>>>(w, g, m, v, static_cast<bf16*>(w16), n, hyper, b1, b2,
                                            eps);
  gdn::count_launches(n > 0 ? 2 : 1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_to_bf16(const float* a, void* b, int64_t n, void* stream) {
  if (!a || !b || n < 0) GDN_BAD_ARG("invalid arguments");
  if (n == 0) return GDN_OK;
  f32_to_bf16<<<blocks_for(n), 256, 0, GDN_S(stream)>>>(a, static_cast<bf16*>(b), n);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}
