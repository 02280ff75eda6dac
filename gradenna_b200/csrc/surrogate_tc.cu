// Surrogate convolutions on the 5th-generation tensor cores (tcgen05).
//
// conv_fwd_tc computes the same implicit-GEMM convolution as conv_fwd
// (surrogate.cu): out[p, co] = act(bias[co] + sum_k im2col(in)[p][k] w[k][co])
// with k = tap * Cin + ci, NHWC bf16 activations (channel slices allowed),
// FP32 accumulation, the same epilogue (bias, leaky ReLU, backward activation
// mask, bf16 / FP32 stores). What differs is the engine:
//
//   * A CTA of 4 warps owns 128 pixels x N output channels (N = 32, 64, 128).
//     The FP32 accumulator tile lives in tensor memory (TMEM, 128 lanes x N
//     columns), allocated by warp 0.
//   * The reduction runs in 64-wide steps. Each step's operands are staged
//     in shared memory in the canonical K-major, 128-byte-swizzled layout the
//     tensor core reads directly: 8-row x 128-byte atoms, the 16-byte chunk
//     c of row r stored at chunk c ^ (r % 8). A is the im2col tile (128
//     pixel rows x 64 reduction indices, gathered with 16-byte cp.async and
//     zero fill at the image border), B the weight tile read from a K-major
//     copy of the weights ([Cout][K]). Three stages are in flight.
//   * One thread issues the MMAs (tcgen05.mma.cta_group::1.kind::f16, M = 128,
//     K = 16 each, four per step) and commits each step to an mbarrier;
//     a stage is refilled only after the MMAs that read it completed.
//   * After the last step each warp reads its 32 TMEM lanes (= 32 pixel rows)
//     with tcgen05.ld and applies the epilogue.
//
// Every mbarrier wait is bounded: when it runs out the kernel records the
// failure in a device flag, drains its own copies, releases TMEM and
// returns without writing results; gdn_sur_status reads (and resets) the
// flag, so a caller can check a batch of launches with one synchronisation.
//
// No reference counterpart (the reference has no learned component).
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"

namespace gdn {
namespace surrtc {

using bf16 = __nv_bfloat16;

constexpr int TM = 128;      // pixels per CTA (UMMA M)
constexpr int TK = 64;       // reduction indices per stage (one 128-byte row)
constexpr int STAGES = 3;
constexpr int THREADS = 128;
constexpr long long WAIT_LIMIT = 1LL << 22;  // mbarrier polls before giving up

__device__ int g_tc_error = 0;
// Test hook: when >= 0, the CTAs of the next launches give up at this
// reduction step as if a stage wait had run out (they wait, bounded, on a
// barrier nothing arrives at), so the abort path can be exercised on purpose.
__device__ int g_tc_inject_step = -1;
constexpr long long INJECT_LIMIT = 1LL << 10;

struct Args {
  const bf16* in;
  int in_stride, in_c0;
  int N, H, W, Cin, taps;
  const bf16* wk;  // [Cout][K], K = taps * Cin
  const float* bias;
  int Cout, relu;
  float slope;
  bf16* out;
  int out_stride, out_c0;
  float* out32;
  const bf16* mask;
  int mask_stride, mask_c0;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(unsigned dst, const void* src, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (stride byte offset), leading byte offset 16 (unused by
// swizzled K-major layouts), descriptor version 1.
__device__ __forceinline__ uint64_t sw128_desc(unsigned addr) {
  return (uint64_t((addr >> 4) & 0x3FFF)) | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32) |
         (uint64_t(1) << 46) | (uint64_t(2) << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
template <int N>
__device__ __forceinline__ uint32_t idesc_bf16() {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(TM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  for (long long i = 0; i < WAIT_LIMIT; ++i)
    if (mbar_try(bar, parity)) return true;
  return false;
}

template <int N>
__global__ void __launch_bounds__(THREADS) conv_fwd_tc(Args a) {
  extern __shared__ __align__(1024) unsigned char dyn[];
  constexpr int A_BYTES = TM * 128;
  constexpr int B_BYTES = N * 128;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  // 1024-byte aligned stage base (the swizzle pattern is tied to address bits)
  const unsigned raw = smem_u32(dyn);
  const unsigned base = (raw + 1023u) & ~1023u;
  __shared__ __align__(8) unsigned long long bars[STAGES + 1];  // + the never-arriving one
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long P = (long long)a.N * a.H * a.W;
  const long long p0 = (long long)blockIdx.x * TM;
  const int n0 = blockIdx.y * N;
  const int K = a.taps * a.Cin;
  const int nk = (K + TK - 1) / TK;

  if (tid == 0) {
    for (int s = 0; s <= STAGES; ++s) mbar_init(smem_u32(&bars[s]), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = tmem_slot;

  // Row of the im2col tile owned by this thread (all 8 chunks of it).
  const long long prow = p0 + tid;
  const bool row_ok = prow < P;
  int pn = 0, py = 0, px = 0;
  if (row_ok) {
    const long long hw = (long long)a.H * a.W;
    pn = int(prow / hw);
    const int rem = int(prow - (long long)pn * hw);
    py = rem / a.W;
    px = rem - py * a.W;
  }

  auto load = [&](int t) {
    const int s = t % STAGES;
    const unsigned sa = base + s * STAGE_BYTES;
    const unsigned sb = sa + A_BYTES;
    const int k0 = t * TK;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int k = k0 + c * 8;
      bool ok = row_ok && k < K;
      const bf16* src = a.in;
      if (ok) {
        const int tap = k / a.Cin, ci = k - tap * a.Cin;
        const int dy = a.taps == 9 ? tap / 3 - 1 : 0, dx = a.taps == 9 ? tap % 3 - 1 : 0;
        const int y = py + dy, x = px + dx;
        ok = y >= 0 && y < a.H && x >= 0 && x < a.W;
        if (ok) src = a.in + (((long long)pn * a.H + y) * a.W + x) * a.in_stride + a.in_c0 + ci;
      }
      cp_async16(sa + tid * 128 + ((c ^ (tid & 7)) << 4), src, ok);
    }
    // B: N rows (output channels) x 8 chunks of 8 reduction indices.
#pragma unroll
    for (int q = tid; q < N * 8; q += THREADS) {
      const int r = q >> 3, c = q & 7;
      const int co = n0 + r, k = k0 + c * 8;
      const bool ok = co < a.Cout && k < K;
      cp_async16(sb + r * 128 + ((c ^ (r & 7)) << 4),
                 ok ? a.wk + (long long)co * K + k : a.wk, ok);
    }
  };

  const int inject = g_tc_inject_step;
  bool failed = false;
  int issued = 0;  // steps whose MMAs have been issued and committed
  // Prologue: stages 0 .. STAGES-2.
  for (int t = 0; t < STAGES - 1; ++t) {
    if (t < nk) load(t);
    asm volatile("cp.async.commit_group;\n" ::);
  }
  for (int c = 0; c < nk; ++c) {
    const int t = c + STAGES - 1;
    if (t < nk) {
      if (t >= STAGES) {
        // Stage t % STAGES was last read by the MMAs of step t - STAGES.
        const int u = t - STAGES;
        if (!mbar_wait(smem_u32(&bars[u % STAGES]), (u / STAGES) & 1)) failed = true;
      }
      if (!failed) load(t);
    }
    if (c == inject && tid == 0) {
      // Nothing arrives at bars[STAGES]: this wait runs out.
      bool ok = false;
      for (long long i = 0; i < INJECT_LIMIT && !ok; ++i) ok = mbar_try(smem_u32(&bars[STAGES]), 0);
      if (!ok) failed = true;
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group %0;\n" ::"n"(STAGES - 1));
    // Make this thread's cp.async writes visible to the tensor core's proxy.
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    if (failed) atomicExch(&abort_flag, 1);
    __syncthreads();
    if (abort_flag) break;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const unsigned sa = base + (c % STAGES) * STAGE_BYTES;
      const unsigned sb = sa + A_BYTES;
      const uint64_t da = sw128_desc(sa), db = sw128_desc(sb);
      const uint32_t id = idesc_bf16<N>();
#pragma unroll
      for (int kk = 0; kk < TK / 16; ++kk) {
        const uint32_t accumulate = (c > 0 || kk > 0) ? 1u : 0u;
        // +32 bytes per K = 16 step inside the swizzled 128-byte row.
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(da + uint64_t(2 * kk)), "l"(db + uint64_t(2 * kk)), "r"(id), "r"(accumulate));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(&bars[c % STAGES])));
    }
    issued = c + 1;
  }
  // Wait for every MMA issued so far, on the normal path and after an abort
  // alike: the last commit tracks all earlier MMAs of the issuing thread, and
  // none may still read shared memory or write TMEM when TMEM is released
  // and the CTA exits. The wait is bounded like the others.
  if (issued > 0) {
    const int u = issued - 1;
    if (!mbar_wait(smem_u32(&bars[u % STAGES]), (u / STAGES) & 1)) atomicExch(&abort_flag, 1);
  }
  asm volatile("cp.async.wait_all;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (abort_flag) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
  } else {
    // Epilogue: warp w holds TMEM lanes 32w .. 32w + 31 = pixel rows.
    const long long p = p0 + warp * 32 + lane;
    const bool pok = p < P;
    // 16-byte vector path when every 16-channel run starts 16-byte aligned.
    const bool vec = (!a.out || (a.out_stride % 8 == 0 && a.out_c0 % 8 == 0 &&
                                 (reinterpret_cast<uintptr_t>(a.out) & 15) == 0)) &&
                     (!a.mask || (a.mask_stride % 8 == 0 && a.mask_c0 % 8 == 0 &&
                                  (reinterpret_cast<uintptr_t>(a.mask) & 15) == 0)) &&
                     (!a.out32 || (a.Cout % 4 == 0 && (reinterpret_cast<uintptr_t>(a.out32) & 15) == 0));
#pragma unroll
    for (int cb = 0; cb < N; cb += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(cb);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
          "%11, %12, %13, %14, %15}, [%16];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
      if (pok && vec && n0 + cb + 16 <= a.Cout) {
        // 16 consecutive channels of one pixel: two 16-byte loads / stores.
        const int co0 = n0 + cb;
        float x[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          x[j] = __uint_as_float(v[j]) + (a.bias ? a.bias[co0 + j] : 0.f);
          if (a.relu && !(x[j] > 0.f)) x[j] *= a.slope;
        }
        if (a.mask) {
          const uint4* mp = reinterpret_cast<const uint4*>(a.mask + p * a.mask_stride + a.mask_c0 + co0);
          const uint4 m0 = mp[0], m1 = mp[1];
          const bf16* mb0 = reinterpret_cast<const bf16*>(&m0);
          const bf16* mb1 = reinterpret_cast<const bf16*>(&m1);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (!(__bfloat162float(mb0[j]) > 0.f)) x[j] *= a.slope;
            if (!(__bfloat162float(mb1[j]) > 0.f)) x[j + 8] *= a.slope;
          }
        }
        if (a.out) {
          uint4 o[2];
          bf16* ob = reinterpret_cast<bf16*>(o);
#pragma unroll
          for (int j = 0; j < 16; ++j) ob[j] = __float2bfloat16(x[j]);
          uint4* dp = reinterpret_cast<uint4*>(a.out + p * a.out_stride + a.out_c0 + co0);
          dp[0] = o[0];
          dp[1] = o[1];
        }
        if (a.out32) {
          float4* dp = reinterpret_cast<float4*>(a.out32 + p * a.Cout + co0);
#pragma unroll
          for (int j = 0; j < 4; ++j) dp[j] = make_float4(x[4 * j], x[4 * j + 1], x[4 * j + 2], x[4 * j + 3]);
        }
      } else if (pok) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int co = n0 + cb + j;
          if (co >= a.Cout) break;
          float x = __uint_as_float(v[j]) + (a.bias ? a.bias[co] : 0.f);
          if (a.relu && !(x > 0.f)) x *= a.slope;
          if (a.mask && !(__bfloat162float(a.mask[p * a.mask_stride + a.mask_c0 + co]) > 0.f))
            x *= a.slope;
          if (a.out) a.out[p * a.out_stride + a.out_c0 + co] = __float2bfloat16(x);
          if (a.out32) a.out32[p * a.Cout + co] = x;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(N));
}

// K-major weights for conv_fwd_tc: wk[co'][k'] of the convolution to run.
// Forward (flip = 0): wk[co][tap * Cin + ci] = w[tap * Cin + ci][co].
// Input gradient (flip = 1; Cin' = Cout, Cout' = Cin):
//   wk[ci][(taps - 1 - tap) * Cout + co] = w[tap * Cin + ci][co].
__global__ void weights_kmajor(const bf16* __restrict__ w, int Cin, int Cout, int taps, int flip,
                               bf16* __restrict__ wk) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)taps * Cin * Cout;
  if (i >= total) return;
  const int co = int(i % Cout);
  const long long kc = i / Cout;
  const int ci = int(kc % Cin), tap = int(kc / Cin);
  if (!flip)
    wk[(long long)co * taps * Cin + kc] = w[i];
  else
    wk[(long long)ci * taps * Cout + (long long)(taps - 1 - tap) * Cout + co] = w[i];
}

template <int N>
int launch(const Args& a, cudaStream_t s) {
  constexpr int smem = STAGES * (TM * 128 + N * 128) + 1024;
  // The dynamic shared-memory limit is a per-device function attribute.
  static bool configured[64] = {};
  int dev = 0;
  GDN_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) GDN_BAD_ARG("device index %d out of range", dev);
  if (!configured[dev]) {
    GDN_TRY_CUDA(cudaFuncSetAttribute(conv_fwd_tc<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
    configured[dev] = true;
  }
  const long long P = (long long)a.N * a.H * a.W;
  const dim3 grid(unsigned((P + TM - 1) / TM), unsigned((a.Cout + N - 1) / N));
  conv_fwd_tc<N><<<grid, THREADS, smem, s>>>(a);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

inline bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace surrtc
}  // namespace gdn

using namespace gdn::surrtc;

extern "C" int gdn_sur_conv_fwd_tc(const void* in, int32_t in_stride, int32_t in_c0, int32_t N,
                                   int32_t H, int32_t W, int32_t Cin, int32_t taps, const void* wk,
                                   const float* bias, int32_t Cout, int32_t relu, float slope,
                                   void* out, int32_t out_stride, int32_t out_c0, float* out32,
                                   const void* mask, int32_t mask_stride, int32_t mask_c0,
                                   void* stream) {
  if (N <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0 || (taps != 1 && taps != 9))
    GDN_BAD_ARG("invalid convolution shape");
  if (!in || !wk || (!out && !out32)) GDN_BAD_ARG("null pointer");
  if (in_c0 < 0 || in_c0 + Cin > in_stride) GDN_BAD_ARG("input channel slice out of range");
  if (out && (out_c0 < 0 || out_c0 + Cout > out_stride)) GDN_BAD_ARG("output channel slice out of range");
  if (mask && (mask_c0 < 0 || mask_c0 + Cout > mask_stride)) GDN_BAD_ARG("mask channel slice out of range");
  // 16-byte staging: every 8-element chunk of a row must start 16-byte aligned.
  if (Cin % 8 || in_stride % 8 || in_c0 % 8 || !al16(in) || !al16(wk))
    GDN_BAD_ARG("tensor-core convolution needs Cin, the input stride and offset multiples of 8 "
                "and 16-byte aligned input and weights");
  Args a{static_cast<const bf16*>(in), in_stride, in_c0, N, H, W, Cin, taps,
         static_cast<const bf16*>(wk), bias, Cout, relu, slope, static_cast<bf16*>(out),
         out_stride, out_c0, out32, static_cast<const bf16*>(mask), mask_stride, mask_c0};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // Channel tile: the smallest of 32 / 64 / 128 covering Cout, narrowed while
  // the grid holds fewer than two CTAs per SM (the coarse U-Net levels have
  // few pixels), since one 128-thread CTA cannot keep an SM's tensor core fed.
  static int sms[64] = {};
  int dev = 0;
  GDN_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) GDN_BAD_ARG("device index %d out of range", dev);
  if (!sms[dev]) GDN_TRY_CUDA(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
  const long long mtiles = ((long long)N * H * W + TM - 1) / TM;
  int n = Cout <= 32 ? 32 : (Cout <= 64 ? 64 : 128);
  while (n > 32 && mtiles * ((Cout + n - 1) / n) < 2LL * sms[dev]) n /= 2;
  if (n == 32) return launch<32>(a, s);
  if (n == 64) return launch<64>(a, s);
  return launch<128>(a, s);
}

extern "C" int gdn_sur_weights_kmajor(const void* w, int32_t Cin, int32_t Cout, int32_t taps,
                                      int32_t flip, void* wk, void* stream) {
  if (!w || !wk || Cin <= 0 || Cout <= 0 || (taps != 1 && taps != 9)) GDN_BAD_ARG("invalid arguments");
  const long long n = (long long)taps * Cin * Cout;
  weights_kmajor<<<unsigned((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(w), Cin, Cout, taps, flip, static_cast<bf16*>(wk));
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

extern "C" int gdn_sur_inject_timeout(int32_t step) {
  GDN_TRY_CUDA(cudaMemcpyToSymbol(g_tc_inject_step, &step, sizeof(int)));
  return GDN_OK;
}

extern "C" int gdn_sur_status(int32_t* timeouts, int32_t reset) {
  if (!timeouts) GDN_BAD_ARG("null pointer");
  int v = 0;
  GDN_TRY_CUDA(cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)));
  *timeouts = v;
  if (reset) {
    const int z = 0;
    GDN_TRY_CUDA(cudaMemcpyToSymbol(g_tc_error, &z, sizeof(int)));
  }
  return GDN_OK;
}
