// 3D Yee FDTD time loop for B200 (sm_100a).
//
// Replaces the reference's fused CPU kernel gradenna_3d_run_f32/_f64
// (rust/src/lib3d.rs:191-828, lib3d_sweeps.rs) and the scan body of
// simulate_3d (src/gradenna/fdtd3d.py:559-679) with the same per-step
// order: H (Hx, Hy, Hz with 6 slab psi) -> Mx/My/Mz -> port Ampere current ->
// Ex (+Jx), Ey (+Jy), Ez (+Jz) with 6 psi -> semi-implicit RVS overwrite of
// the port edge -> DFT -> probes / V / energy.
//
// B200 design: two kernels per step updating in place (the H kernel reads
// only E and the E kernel only H, so no CTA ever reads a value another CTA is
// writing). A CTA covers an 8 x 32 (j, k) tile with k contiguous, so every
// field access is a coalesced row, and walks 8 consecutive i-planes. Each
// thread loads all operands of its cell before updating it. CPML psi lives
// in full padded volumes (zero outside the slabs) indexed like the fields;
// only slab cells touch them, on per-thread slab flags. Point work (sources,
// the port, probes) is binned by plane box on the host and applied by the
// owning CTA after its sweep; per plane-box flags keep the other boxes on the
// bare stencil. The running DFT uses the monitor ring of the 2D path: after
// each half step a gather kernel copies the monitored cells to ring slot
// n % R, and one fold kernel per R steps adds sum_t ph[t,k] x_t to the
// accumulators. One chunk of R steps is captured as a CUDA graph and
// replayed; kernels read the absolute step from a counter.
#include <algorithm>
#include <array>
#include <cmath>

#include "common.cuh"

namespace gdn {
namespace yee3d {

constexpr int BK = 32, BJ = 8;  // CTA box along k and j (one i-plane)
constexpr int NT = BK * BJ;
constexpr int KMAX = 16;
constexpr int NC = 6;  // components: ex ey ez hx hy hz

struct Pt3 {
  int m, i, j, k;
};

// A source point applied by the injection kernels: channel (0 Jz, 1 Jx,
// 2 Jy, 3 Mx, 4 My, 5 Mz), index in its channel, cell offset in its field.
struct Fp {
  int type, m;
  long long off;
};

constexpr int MAXF = 64;  // monitors whose offsets the fold stages in shared memory

struct Mon3 {
  int comp, lo0, lo1, lo2, s0, s1, s2, pad;
  long long count, off;
  void* out;
};

template <typename T>
struct Dev3 {
  int nx, ny, nz, npml, n_steps, n_freq, R, gj, gk;  // gj, gk: CTA grid along j, k
  int sy, sz;          // padded strides: cell (i,j,k) at ((i+1)*sy + (j+1))*sz + (k+1)
  long long vol;       // elements per padded volume
  T* f[NC];            // fields
  T* psi;              // 12 padded volumes (see psi_* constants)
  const T *ca, *cb, *eps;  // caller (nx, ny, nz)
  const T *ik_e[3], *ik_h[3];
  const T *be_lo[3], *ce_lo[3], *be_hi[3], *ce_hi[3];
  const T *bh_lo[3], *ch_lo[3], *bh_hi[3], *ch_hi[3];
  T dt_mu, inv_d[3], dx, dy, dz, a_port, b_port, c_port;
  int n_src, n_jx, n_jy, n_mx, n_my, n_mz, n_probes, has_port, pi, pj, pk;
  int port_cta;
  const int* off[7];  // per point type CSR over CTAs: src jx jy mx my mz probe
  const Pt3* pts[7];
  // Source points outside the boxes that hold probes or the port, applied by
  // yee_inject after the half step (side 0 = E sources, 1 = H sources).
  const Fp* fpts[2];
  long long n_fp[2];
  const T *cb_src, *cb_jx, *cb_jy;
  const T* cur[6];  // src jx jy mx my mz
  const T* port_vs;
  int cw;
  const double* cw_env;
  const double2* w[6];
  const double2 *ph_e, *ph_h;
  T *out_probe, *out_v, *out_i;
  const int* pcomp;  // E component of each probe (0 ex, 1 ey, 2 ez), or null = Ez
  T* mring;
  long long mon_cells;
  int n_mons;
  const Mon3* mons;
  // Ring gathers: the ring holds the E-side monitors' cells first (gcells[0]
  // of them), then the H-side ones (gcells[1]); gsrc[r] is the offset of
  // ring cell r's field value in the contiguous block of the six fields
  // (32-bit when the block holds fewer than 2^32 values, else gsrc64).
  const unsigned* gsrc;
  const long long* gsrc64;
  long long gcells[2];
  const unsigned char* cls;  // per plane-box work flags (F_*)
  T* cwv;                // CW source values of the chunk: [sub][cw_off[type] + m]
  long long cw_total, cw_off[6];
  const int* step_base;
};

// psi volume order: field x stretched axis.
enum { P_EXY, P_EXZ, P_EYX, P_EYZ, P_EZX, P_EZY, P_HXY, P_HXZ, P_HYX, P_HYZ, P_HZX, P_HZY };

template <typename T>
__device__ __forceinline__ long long at(const Dev3<T>& d, int i, int j, int k) {
  return ((long long)(i + 1) * d.sy + (j + 1)) * d.sz + (k + 1);
}

// Source value of point m of channel `type` at step n (chunk offset sub):
// tabulated, or the chunk's CW values synthesised by yee_cw_synth.
template <typename T>
__device__ __forceinline__ T wave(const Dev3<T>& d, int type, int n_pts, int m, int n, int sub) {
  if (d.cw) return d.cwv[(long long)sub * d.cw_total + d.cw_off[type] + m];
  return d.cur[type][(long long)n * n_pts + m];
}

// CW source values J(n) = env[n] Re(sum_k W_k conj(ph[n,k])) of every point
// for the `cnt` steps of a chunk, once per chunk instead of once per step.
// The chunk's phase rows are staged in shared memory and each point's K
// weights are held in registers.
template <typename T>
__global__ void __launch_bounds__(256) yee_cw_synth(Dev3<T> d, int cnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* sph = reinterpret_cast<double2*>(smem_raw);  // [2][cnt][K]: E-type, H-type
  const int n0 = *d.step_base, K = d.n_freq;
  for (int q = threadIdx.x; q < cnt * K; q += blockDim.x) {
    sph[q] = d.ph_e[(long long)n0 * K + q];
    sph[cnt * K + q] = d.ph_h[(long long)n0 * K + q];
  }
  __syncthreads();
  const long long mg = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (mg >= d.cw_total) return;
  int type = 0;
#pragma unroll
  for (int t = 1; t < 6; ++t)
    if (mg >= d.cw_off[t]) type = t;
  const long long m = mg - d.cw_off[type];
  const double2* w = d.w[0];
#pragma unroll
  for (int t = 1; t < 6; ++t)
    if (type == t) w = d.w[t];
  const double2* ph = sph + (type <= 2 ? 0 : cnt * K);
  double2 wr[KMAX];
#pragma unroll
  for (int k = 0; k < KMAX; ++k) wr[k] = k < K ? w[m * K + k] : make_double2(0.0, 0.0);
  for (int t = 0; t < cnt; ++t) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < KMAX; ++k)
      if (k < K) {
        const double2 p = ph[t * K + k];
        s += wr[k].x * p.x + wr[k].y * p.y;
      }
    d.cwv[(long long)t * d.cw_total + mg] = T(d.cw_env[n0 + t] * s);
  }
}

// Programmatic dependent launch: the step and injection kernels of a chunk
// are launched with programmatic stream serialisation, so the next kernel's
// CTAs are scheduled as this kernel's CTAs drain instead of after a full
// launch round trip. Every such kernel first waits until its predecessor
// grid has completed and its writes are visible (griddepcontrol.wait, a
// no-op for a normal launch), then allows its own dependents to launch.
__device__ __forceinline__ void dependent_launch_gate() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// Source injection after a half step (fdtd3d.py:585-588 for Mx/My/Mz,
// 606-622 for Jx/Jy/Jz): one thread per source point that no step-kernel
// CTA handles, E = E - c_b,src J or H = H - (dt/mu) M. The step kernels
// keep only the points of boxes that also hold probes or the port, which
// must see the source before they read the field; everything else would
// put a barrier and a point loop into most plane boxes (the adjoint run
// drives every NTFF face cell).
template <typename T>
__global__ void __launch_bounds__(256) yee_inject(Dev3<T> d, int sub, int side) {
  dependent_launch_gate();
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.n_fp[side]) return;
  const Fp p = d.fpts[side][r];
  const int n = *d.step_base + sub;
  const int counts[6] = {d.n_src, d.n_jx, d.n_jy, d.n_mx, d.n_my, d.n_mz};
  const T v = wave(d, p.type, counts[p.type], p.m, n, sub);
  T coef;
  int comp;
  if (p.type == 0) {
    coef = d.cb_src[p.m];
    comp = 2;
  } else if (p.type == 1) {
    coef = d.cb_jx[p.m];
    comp = 0;
  } else if (p.type == 2) {
    coef = d.cb_jy[p.m];
    comp = 1;
  } else {
    coef = d.dt_mu;
    comp = p.type;  // 3 hx, 4 hy, 5 hz
  }
  atomicAdd(d.f[comp] + p.off, -(coef * v));
}

// Monitor ring writes of step n (fdtd3d.py:635-662, the running DFT's
// samples): after the H (side 1) or the E (side 0) half step, one thread per
// monitored cell of that side copies the field value into ring slot n % R,
// through a table of field offsets built once on the host.
// Doing this in its own launch keeps the per-cell stencil kernels free of
// monitor bookkeeping; the ring traffic is O(monitored cells).
template <typename T>
__global__ void __launch_bounds__(256) yee_gather(Dev3<T> d, int sub, int side) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.gcells[side]) return;
  const long long at_r = (side ? d.gcells[0] : 0) + r;
  const int n = *d.step_base + sub;
  const long long src = d.gsrc ? (long long)d.gsrc[at_r] : d.gsrc64[at_r];
  d.mring[(long long)(n % d.R) * d.mon_cells + at_r] = d.f[0][src];
}

// Per plane-box flags (bit set = the box needs that work), computed on the
// host so that most boxes run the bare stencil with no per-thread checks.
enum : unsigned char { F_HPTS = 1, F_EPTS = 2, F_CPML = 8 };

// A CTA walks `ni` consecutive i-planes of its (j, k) tile (chosen on the
// host, planes_per_cta).

// CPML coefficients of sample s of axis ax (E-type: the ns = n-2 samples
// of the PEC interior; H-type: the ns = n-1 half samples). Returns whether
// s lies in a slab; outside, b = c = 0 and 1/kappa = 1 (cpml.py:161-208).
template <typename T, bool E>
__device__ __forceinline__ bool slab_coef(const Dev3<T>& d, int ax, int s, int ns, T& b, T& c,
                                          T& ik) {
  const int m = d.npml;
  b = T(0);
  c = T(0);
  ik = T(1);
  if (s < 0 || s >= ns) return false;
  if (s < m) {
    b = E ? d.be_lo[ax][s] : d.bh_lo[ax][s];
    c = E ? d.ce_lo[ax][s] : d.ch_lo[ax][s];
    ik = E ? d.ik_e[ax][s] : d.ik_h[ax][s];
    return true;
  }
  if (s >= ns - m) {
    const int t = s - (ns - m);
    b = E ? d.be_hi[ax][t] : d.bh_hi[ax][t];
    c = E ? d.ce_hi[ax][t] : d.ch_hi[ax][t];
    ik = E ? d.ik_e[ax][s] : d.ik_h[ax][s];
    return true;
  }
  return false;
}

// One axis' CPML state of a thread: whether its sample is in a slab and the
// coefficients there.
template <typename T>
struct Ax {
  bool on;
  T b, c, ik;
};

// psi <- b psi + c diff; the term diff/kappa + psi (cpml.py:120-158).
template <typename T>
__device__ __forceinline__ T psi_term(const Ax<T>& a, T diff, T& psi) {
  psi = a.b * psi + a.c * diff;
  return diff * a.ik + psi;
}

// ---------------------------------------------------------------------------
// H update: E^n -> H^{n+1/2} (fdtd3d.py:564-588) + Mx/My/Mz + H monitors.
// A CTA covers a BJ x BK tile of NI consecutive i-planes.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 5 : 3) yee_h(Dev3<T> d, int sub, int ni) {
  dependent_launch_gate();
  const int n = *d.step_base + sub;
  const int k = blockIdx.x * BK + threadIdx.x;
  const int j = blockIdx.y * BJ + threadIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const bool live = j < ny && k < nz;
  const int tid = threadIdx.y * BK + threadIdx.x;
  const int i0 = int(blockIdx.z) * ni, i1 = min(nx, i0 + ni);
  // 32-bit cell offsets (a padded volume holds fewer than 2^31 cells).
  const int di = d.sy * d.sz, dj = d.sz;
  int c = ((i0 + 1) * d.sy + (j + 1)) * d.sz + (k + 1);
  const T* __restrict__ ex = d.f[0];
  const T* __restrict__ ey = d.f[1];
  const T* __restrict__ ez = d.f[2];
  T *hx = d.f[3], *hy = d.f[4], *hz = d.f[5];
  T *pxz = d.psi + P_HXZ * d.vol, *pxy = d.psi + P_HXY * d.vol, *pyx = d.psi + P_HYX * d.vol,
    *pyz = d.psi + P_HYZ * d.vol, *pzy = d.psi + P_HZY * d.vol, *pzx = d.psi + P_HZX * d.vol;
  const T dt_mu = d.dt_mu, idx = d.inv_d[0], idy = d.inv_d[1], idz = d.inv_d[2];
  // This thread's y and z CPML samples (H-type) are fixed over the planes.
  Ax<T> ay, az;
  ay.on = slab_coef<T, false>(d, 1, j, ny - 1, ay.b, ay.c, ay.ik);
  az.on = slab_coef<T, false>(d, 2, k, nz - 1, az.b, az.c, az.ik);
  const bool vx = j < ny - 1 && k < nz - 1, kin = k < nz - 1, jin = j < ny - 1;
  // Ey and Ez of plane i + 1 become plane i + 1's own values next iteration.
  T ey0 = T(0), ez0 = T(0);
  if (live) {
    ey0 = ey[c];
    ez0 = ez[c];
  }
  for (int i = i0; i < i1; ++i, c += di) {
    const int cta = (i * d.gj + blockIdx.y) * d.gk + blockIdx.x;
    const unsigned fl = d.cls[cta];
    if (live && !(fl & F_CPML)) {
      // No slab within reach of this plane box: the bare update.
      const T ex0 = ex[c];
      const T eyk = ey[c + 1], ezj = ez[c + dj], ezi = ez[c + di];
      const T exk = ex[c + 1], exj = ex[c + dj], eyi = ey[c + di];
      const T hx0 = hx[c], hy0 = hy[c], hz0 = hz[c];
      const bool vy = i < nx - 1 && kin, vz = i < nx - 1 && jin;
      if (vx) hx[c] = hx0 + dt_mu * ((eyk - ey0) * idz - (ezj - ez0) * idy);
      if (vy) hy[c] = hy0 + dt_mu * ((ezi - ez0) * idx - (exk - ex0) * idz);
      if (vz) hz[c] = hz0 + dt_mu * ((exj - ex0) * idy - (eyi - ey0) * idx);
      ey0 = eyi;
      ez0 = ezi;
    } else if (live) {
      Ax<T> ax;
      ax.on = slab_coef<T, false>(d, 0, i, nx - 1, ax.b, ax.c, ax.ik);
      // Every operand first (all in the padded volumes), then the updates.
      const T ex0 = ex[c];
      const T eyk = ey[c + 1], ezj = ez[c + dj], ezi = ez[c + di];
      const T exk = ex[c + 1], exj = ex[c + dj], eyi = ey[c + di];
      const T hx0 = hx[c], hy0 = hy[c], hz0 = hz[c];
      const bool vy = i < nx - 1 && kin, vz = i < nx - 1 && jin;
      T p_xz = T(0), p_xy = T(0), p_yx = T(0), p_yz = T(0), p_zy = T(0), p_zx = T(0);
      if (vx && az.on) p_xz = pxz[c];
      if (vx && ay.on) p_xy = pxy[c];
      if (vy && ax.on) p_yx = pyx[c];
      if (vy && az.on) p_yz = pyz[c];
      if (vz && ay.on) p_zy = pzy[c];
      if (vz && ax.on) p_zx = pzx[c];
      if (vx) {  // Hx (nx, ny-1, nz-1): +dt/mu (t_hxz - t_hxy)
        const T dey_dz = (eyk - ey0) * idz, dez_dy = (ezj - ez0) * idy;
        T tz = dey_dz, ty = dez_dy;
        if (az.on) {
          tz = psi_term(az, dey_dz, p_xz);
          pxz[c] = p_xz;
        }
        if (ay.on) {
          ty = psi_term(ay, dez_dy, p_xy);
          pxy[c] = p_xy;
        }
        hx[c] = hx0 + dt_mu * (tz - ty);
      }
      if (vy) {  // Hy (nx-1, ny, nz-1): +dt/mu (t_hyx - t_hyz)
        const T dez_dx = (ezi - ez0) * idx, dex_dz = (exk - ex0) * idz;
        T tx = dez_dx, tz = dex_dz;
        if (ax.on) {
          tx = psi_term(ax, dez_dx, p_yx);
          pyx[c] = p_yx;
        }
        if (az.on) {
          tz = psi_term(az, dex_dz, p_yz);
          pyz[c] = p_yz;
        }
        hy[c] = hy0 + dt_mu * (tx - tz);
      }
      if (vz) {  // Hz (nx-1, ny-1, nz): +dt/mu (t_hzy - t_hzx)
        const T dex_dy = (exj - ex0) * idy, dey_dx = (eyi - ey0) * idx;
        T ty = dex_dy, tx = dey_dx;
        if (ay.on) {
          ty = psi_term(ay, dex_dy, p_zy);
          pzy[c] = p_zy;
        }
        if (ax.on) {
          tx = psi_term(ax, dey_dx, p_zx);
          pzx[c] = p_zx;
        }
        hz[c] = hz0 + dt_mu * (ty - tx);
      }
      ey0 = eyi;
      ez0 = ezi;
    }
    if (fl & F_HPTS) {
      __syncthreads();
      T* hs[3] = {hx, hy, hz};
      for (int t = 3; t < 6; ++t) {
        const int np_ = t == 3 ? d.n_mx : (t == 4 ? d.n_my : d.n_mz);
        for (int q = d.off[t][cta] + tid; q < d.off[t][cta + 1]; q += NT) {
          const Pt3 p = d.pts[t][q];
          atomicAdd(hs[t - 3] + at(d, p.i, p.j, p.k), -(dt_mu * wave(d, t, np_, p.m, n, sub)));
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// E update: H^{n+1/2} -> E^{n+1} (fdtd3d.py:596-633) + sources, port,
// probes, V/I and E monitors. Same CTA geometry as yee_h.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 5 : 3) yee_e(Dev3<T> d, int sub, int ni) {
  __shared__ T s_port[3];  // Ez^n, curl_z and the plain-updated Ez at the port edge
  dependent_launch_gate();
  const int n = *d.step_base + sub;
  const int k = blockIdx.x * BK + threadIdx.x;
  const int j = blockIdx.y * BJ + threadIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const bool live = j < ny && k < nz;
  const int tid = threadIdx.y * BK + threadIdx.x;
  const int i0 = int(blockIdx.z) * ni, i1 = min(nx, i0 + ni);
  const int di = d.sy * d.sz, dj = d.sz;
  int c = ((i0 + 1) * d.sy + (j + 1)) * d.sz + (k + 1);
  long long g = ((long long)i0 * ny + j) * nz + k;  // node coefficients
  const long long dgi = (long long)ny * nz;
  T *ex = d.f[0], *ey = d.f[1], *ez = d.f[2];
  const T* __restrict__ hx = d.f[3];
  const T* __restrict__ hy = d.f[4];
  const T* __restrict__ hz = d.f[5];
  T *pxy = d.psi + P_EXY * d.vol, *pxz = d.psi + P_EXZ * d.vol, *pyz = d.psi + P_EYZ * d.vol,
    *pyx = d.psi + P_EYX * d.vol, *pzx = d.psi + P_EZX * d.vol, *pzy = d.psi + P_EZY * d.vol;
  const T idx = d.inv_d[0], idy = d.inv_d[1], idz = d.inv_d[2];
  // E-type samples of this thread's y and z (the PEC interior, node - 1).
  Ax<T> ay, az;
  ay.on = slab_coef<T, true>(d, 1, j - 1, ny - 2, ay.b, ay.c, ay.ik);
  az.on = slab_coef<T, true>(d, 2, k - 1, nz - 2, az.b, az.c, az.ik);
  const bool jx = j >= 1 && j <= ny - 2, kx = k >= 1 && k <= nz - 2;
  const bool vx_jk = jx && kx, vy_jk = j < ny - 1 && kx, vz_jk = jx && k < nz - 1;
  // Hy and Hz of plane i - 1 (the previous plane's own values).
  T hyi = T(0), hzi = T(0);
  if (live) {
    hyi = hy[c - di];
    hzi = hz[c - di];
  }
  for (int i = i0; i < i1; ++i, c += di, g += dgi) {
    const int cta = (i * d.gj + blockIdx.y) * d.gk + blockIdx.x;
    const unsigned fl = d.cls[cta];
    const bool port_here = d.has_port && cta == d.port_cta;
    if (live && !(fl & F_CPML)) {
      // No slab within reach of this plane box: the bare update.
      const T hx0 = hx[c], hy0 = hy[c], hz0 = hz[c];
      const T hzj = hz[c - dj], hyk = hy[c - 1], hxk = hx[c - 1], hxj = hx[c - dj];
      const T ex0 = ex[c], ey0 = ey[c], ez0 = ez[c];
      const T ca = d.ca[g], cb = d.cb[g];
      const bool iin = i >= 1 && i <= nx - 2;
      const bool vx = i < nx - 1 && vx_jk, vy = iin && vy_jk, vz = iin && vz_jk;
      if (vx) ex[c] = ca * ex0 + cb * ((hz0 - hzj) * idy - (hy0 - hyk) * idz);
      if (vy) ey[c] = ca * ey0 + cb * ((hx0 - hxk) * idz - (hz0 - hzi) * idx);
      if (vz) {
        const T curl = (hy0 - hyi) * idx - (hx0 - hxj) * idy;
        const T upd = ca * ez0 + cb * curl;
        if (port_here && i == d.pi && j == d.pj && k == d.pk) {
          s_port[0] = ez0;
          s_port[1] = curl;
          s_port[2] = upd;
        }
        ez[c] = upd;
      }
      hyi = hy0;
      hzi = hz0;
    } else if (live) {
      Ax<T> ax;
      ax.on = slab_coef<T, true>(d, 0, i - 1, nx - 2, ax.b, ax.c, ax.ik);
      const T hx0 = hx[c], hy0 = hy[c], hz0 = hz[c];
      const T hzj = hz[c - dj], hyk = hy[c - 1], hxk = hx[c - 1], hxj = hx[c - dj];
      const T ex0 = ex[c], ey0 = ey[c], ez0 = ez[c];
      const T ca = d.ca[g], cb = d.cb[g];
      const bool iin = i >= 1 && i <= nx - 2;
      const bool vx = i < nx - 1 && vx_jk, vy = iin && vy_jk, vz = iin && vz_jk;
      T p_xy = T(0), p_xz = T(0), p_yz = T(0), p_yx = T(0), p_zx = T(0), p_zy = T(0);
      if (vx && ay.on) p_xy = pxy[c];
      if (vx && az.on) p_xz = pxz[c];
      if (vy && az.on) p_yz = pyz[c];
      if (vy && ax.on) p_yx = pyx[c];
      if (vz && ax.on) p_zx = pzx[c];
      if (vz && ay.on) p_zy = pzy[c];
      if (vx) {  // Ex (nx-1, ny, nz) interior j, k: t_exy - t_exz
        const T dhz_dy = (hz0 - hzj) * idy, dhy_dz = (hy0 - hyk) * idz;
        T ty = dhz_dy, tz = dhy_dz;
        if (ay.on) {
          ty = psi_term(ay, dhz_dy, p_xy);
          pxy[c] = p_xy;
        }
        if (az.on) {
          tz = psi_term(az, dhy_dz, p_xz);
          pxz[c] = p_xz;
        }
        ex[c] = ca * ex0 + cb * (ty - tz);
      }
      if (vy) {  // Ey (nx, ny-1, nz) interior i, k: t_eyz - t_eyx
        const T dhx_dz = (hx0 - hxk) * idz, dhz_dx = (hz0 - hzi) * idx;
        T tz = dhx_dz, tx = dhz_dx;
        if (az.on) {
          tz = psi_term(az, dhx_dz, p_yz);
          pyz[c] = p_yz;
        }
        if (ax.on) {
          tx = psi_term(ax, dhz_dx, p_yx);
          pyx[c] = p_yx;
        }
        ey[c] = ca * ey0 + cb * (tz - tx);
      }
      if (vz) {  // Ez (nx, ny, nz-1) interior i, j: t_ezx - t_ezy
        const T dhy_dx = (hy0 - hyi) * idx, dhx_dy = (hx0 - hxj) * idy;
        T tx = dhy_dx, ty = dhx_dy;
        if (ax.on) {
          tx = psi_term(ax, dhy_dx, p_zx);
          pzx[c] = p_zx;
        }
        if (ay.on) {
          ty = psi_term(ay, dhx_dy, p_zy);
          pzy[c] = p_zy;
        }
        const T curl = tx - ty;
        const T upd = ca * ez0 + cb * curl;
        if (port_here && i == d.pi && j == d.pj && k == d.pk) {
          s_port[0] = ez0;
          s_port[1] = curl;
          s_port[2] = upd;
        }
        ez[c] = upd;
      }
      hyi = hy0;
      hzi = hz0;
    }
    if (fl & F_EPTS) {
      __syncthreads();
      T* es[3] = {ez, ex, ey};  // point types 0 src (Jz), 1 jx, 2 jy
      const T* cbs[3] = {d.cb_src, d.cb_jx, d.cb_jy};
      const int nps[3] = {d.n_src, d.n_jx, d.n_jy};
      for (int t = 0; t < 3; ++t)
        for (int q = d.off[t][cta] + tid; q < d.off[t][cta + 1]; q += NT) {
          const Pt3 p = d.pts[t][q];
          atomicAdd(es[t] + at(d, p.i, p.j, p.k), -(cbs[t][p.m] * wave(d, t, nps[t], p.m, n, sub)));
        }
      __syncthreads();
      if (port_here && tid == 0) {
        const long long cp = at(d, d.pi, d.pj, d.pk);
        // A current source on the port edge enters the port's semi-implicit
        // update like the curl does: its plain increment (ez - upd, added by
        // the source loop above) rescaled from c_b to the port's b.
        const T src = ez[cp] - s_port[2];
        const T ez_new = d.a_port * s_port[0] + d.b_port * s_port[1] + d.c_port * d.port_vs[n] +
                         (src != T(0) ? src * (d.b_port / d.cb[((long long)d.pi * ny + d.pj) * nz + d.pk]) : T(0));
        ez[cp] = ez_new;
        d.out_v[n] = T(-0.5) * d.dz * (s_port[0] + ez_new);
        d.out_i[n] = (hy[cp] - hy[cp - di]) * d.dy + (hx[cp - dj] - hx[cp]) * d.dx;
      }
      __syncthreads();
      for (int q = d.off[6][cta] + tid; q < d.off[6][cta + 1]; q += NT) {
        const Pt3 p = d.pts[6][q];
        const T* pf = d.pcomp ? d.f[d.pcomp[p.m]] : ez;
        d.out_probe[(long long)n * d.n_probes + p.m] = pf[at(d, p.i, p.j, p.k)];
      }
    }
  }
}

// DFT fold over `cnt` ring slots (fdtd3d.py:635-662).
template <typename T, typename A, int KM>
__global__ void __launch_bounds__(256) yee_fold(Dev3<T> d, int cnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* sph = reinterpret_cast<A*>(smem_raw);
  using C = typename Cplx<A>::type;
  const int n0 = *d.step_base;
  const int K = d.n_freq;
  for (int idx = threadIdx.x; idx < cnt * K; idx += blockDim.x) {
    const int t = idx / K, kk = idx - t * K;
    const double2 pe = d.ph_e[(long long)(n0 + t) * K + kk];
    const double2 ph = d.ph_h[(long long)(n0 + t) * K + kk];
    sph[2 * idx] = A(pe.x);
    sph[2 * idx + 1] = A(pe.y);
    sph[2 * (cnt * K + idx)] = A(ph.x);
    sph[2 * (cnt * K + idx) + 1] = A(ph.y);
  }
  __syncthreads();
  __shared__ long long sOff[MAXF];
  const int nm = d.n_mons;
  if (nm <= MAXF)
    for (int m = threadIdx.x; m < nm; m += blockDim.x) sOff[m] = d.mons[m].off;
  __syncthreads();
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.mon_cells) return;
  int lo = 0, hi = nm - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const long long o = nm <= MAXF ? sOff[mid] : d.mons[mid].off;
    if (o <= r)
      lo = mid;
    else
      hi = mid - 1;
  }
  const Mon3 mon = d.mons[lo];
  const long long loc = r - mon.off;
  const A* ph = sph + (mon.comp < 3 ? 0 : 2 * cnt * K);
  A are[KM], aim[KM];
#pragma unroll
  for (int kk = 0; kk < KM; ++kk) are[kk] = aim[kk] = A(0);
  const T* base = d.mring + r;
  int slot = n0 % d.R;
  for (int t0 = 0; t0 < cnt; t0 += 8) {
    A x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      x[u] = A(0);
      if (t0 + u < cnt) {
        const int sl = slot + u >= d.R ? slot + u - d.R : slot + u;
        x[u] = A(base[(long long)sl * d.mon_cells]);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      if (t0 + u < cnt) {
        const A* pt = ph + 2 * (t0 + u) * K;
#pragma unroll
        for (int kk = 0; kk < KM; ++kk)
          if (kk < K) {
            are[kk] += pt[2 * kk] * x[u];
            aim[kk] += pt[2 * kk + 1] * x[u];
          }
      }
    }
    slot += 8;
    if (slot >= d.R) slot -= d.R;
  }
  C* acc = static_cast<C*>(mon.out) + loc;
#pragma unroll
  for (int kk = 0; kk < KM; ++kk)
    if (kk < K) {
      C v = acc[(long long)kk * mon.count];
      v.x += are[kk];
      v.y += aim[kk];
      acc[(long long)kk * mon.count] = v;
    }
}

// Total field energy (fdtd3d.py:171-183) of the state after step n.
template <typename T>
__global__ void yee_energy(Dev3<T> d, double* eacc, int sub) {
  const int n = *d.step_base + sub;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  double ue = 0.0, uh = 0.0;
  const long long total = (long long)nx * ny * nz;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = int(g / ((long long)ny * nz));
    const int rem = int(g - (long long)i * ny * nz);
    const int j = rem / nz, k = rem - j * nz;
    const long long c = at(d, i, j, k);
    const double ep = double(d.eps[g]);
    const double a = double(d.f[0][c]), b = double(d.f[1][c]), e = double(d.f[2][c]);
    ue += ep * (a * a + b * b + e * e);  // components are zero outside their grids
    const double x = double(d.f[3][c]), y = double(d.f[4][c]), z = double(d.f[5][c]);
    uh += x * x + y * y + z * z;
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
__global__ void yee_energy_finish(const double* eacc, T* out, int n_steps, double cell, double mu0) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < n_steps) out[n] = T(0.5 * cell * eacc[2 * n] + 0.5 * mu0 * cell * eacc[2 * n + 1]);
}

__global__ void yee_advance(int* step_base, int cnt) { *step_base += cnt; }

// Final fields into the caller's unpadded component arrays.
template <typename T>
__global__ void yee_copy_out(Dev3<T> d, T* e0, T* e1, T* e2, T* h0, T* h1, T* h2) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const long long total = (long long)nx * ny * nz;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = int(g / ((long long)ny * nz));
    const int rem = int(g - (long long)i * ny * nz);
    const int j = rem / nz, k = rem - j * nz;
    const long long c = at(d, i, j, k);
    if (i < nx - 1) e0[((long long)i * ny + j) * nz + k] = d.f[0][c];
    if (j < ny - 1) e1[((long long)i * (ny - 1) + j) * nz + k] = d.f[1][c];
    if (k < nz - 1) e2[((long long)i * ny + j) * (nz - 1) + k] = d.f[2][c];
    if (j < ny - 1 && k < nz - 1) h0[((long long)i * (ny - 1) + j) * (nz - 1) + k] = d.f[3][c];
    if (i < nx - 1 && k < nz - 1) h1[((long long)i * ny + j) * (nz - 1) + k] = d.f[4][c];
    if (i < nx - 1 && j < ny - 1) h2[((long long)i * (ny - 1) + j) * nz + k] = d.f[5][c];
  }
}

template <typename C>
__global__ void yee_dft_scale(C* a, long long count, double s) {
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

static void comp_shape(int c, int nx, int ny, int nz, int s[3]) {
  const int sh[6][3] = {{nx - 1, ny, nz},     {nx, ny - 1, nz},     {nx, ny, nz - 1},
                        {nx, ny - 1, nz - 1}, {nx - 1, ny, nz - 1}, {nx - 1, ny - 1, nz}};
  for (int a = 0; a < 3; ++a) s[a] = sh[c][a];
}

struct Layout3 {
  int sy = 0, sz = 0, gj = 0, gk = 0, n_cta = 0, R = 32;
  long long vol = 0, mon_cells = 0;
  size_t fields, psi, zero_end, off[7], pts[7], pcomp, fpts, mons, gsrc, mring, step, eacc, cwv,
      cls, total;
};

// Monitor boxes {comp, lo0, lo1, lo2, s0, s1, s2} in ring order: the listed
// boxes, or the six full components when none are listed.
static std::vector<std::array<int, 7>> mon_boxes3(const GdnYeeParams* p,
                                                  const GdnYeePoints* pts) {
  std::vector<std::array<int, 7>> v;
  if (p->n_freq <= 0) return v;
  if (p->n_monitors == 0) {
    for (int c = 0; c < 6; ++c) {
      int s[3];
      comp_shape(c, p->nx, p->ny, p->nz, s);
      v.push_back({c, 0, 0, 0, s[0], s[1], s[2]});
    }
    return v;
  }
  for (int k = 0; k < p->n_monitors; ++k) {
    const GdnDftMonitor& g = pts->monitors[k];
    v.push_back({g.comp, g.lo[0], g.lo[1], g.lo[2], g.hi[0] - g.lo[0], g.hi[1] - g.lo[1],
                 g.hi[2] - g.lo[2]});
  }
  return v;
}

static long long mon_cells3(const GdnYeeParams* p, const GdnYeePoints* pts) {
  if (p->n_freq <= 0) return 0;
  long long c = 0;
  if (p->n_monitors == 0) {
    for (int k = 0; k < 6; ++k) {
      int s[3];
      comp_shape(k, p->nx, p->ny, p->nz, s);
      c += (long long)s[0] * s[1] * s[2];
    }
    return c;
  }
  for (int k = 0; k < p->n_monitors; ++k) {
    const GdnDftMonitor& m = pts->monitors[k];
    c += (long long)(m.hi[0] - m.lo[0]) * (m.hi[1] - m.lo[1]) * (m.hi[2] - m.lo[2]);
  }
  return c;
}

static const int32_t* pts_of(const GdnYeePoints* pts, int t) {
  const int32_t* a[7] = {pts->src, pts->jx, pts->jy, pts->mx, pts->my, pts->mz, pts->probe};
  return a[t];
}
static int count_of(const GdnYeeParams* p, int t) {
  const int a[7] = {p->n_src, p->n_jx, p->n_jy, p->n_mx, p->n_my, p->n_mz, p->n_probes};
  return a[t];
}

static Layout3 make_layout3(const GdnYeeParams* p, const GdnYeePoints* pts, size_t esize) {
  Layout3 L;
  L.sz = int(div_up(p->nz + 2, 4) * 4);
  L.sy = p->ny + 2;
  L.vol = (long long)(p->nx + 2) * L.sy * L.sz;
  L.gk = int(div_up(p->nz, BK));
  L.gj = int(div_up(p->ny, BJ));
  L.n_cta = p->nx * L.gj * L.gk;
  L.mon_cells = pts ? mon_cells3(p, pts) : 0;
  const size_t budget = size_t(2) << 30;
  long long r = L.mon_cells > 0 ? (long long)(budget / (size_t(L.mon_cells) * esize)) : 32;
  L.R = int(std::max<long long>(1, std::min<long long>(32, r)));
  Carve cv;
  L.fields = cv.take<char>(size_t(NC) * L.vol * esize);
  L.psi = cv.take<char>(size_t(12) * L.vol * esize);
  L.step = cv.take<int>(1);
  L.zero_end = cv.take<char>(0);
  for (int t = 0; t < 7; ++t) {
    L.off[t] = cv.take<int>(L.n_cta + 1);
    L.pts[t] = cv.take<Pt3>(std::max(count_of(p, t), 1));
  }
  L.pcomp = cv.take<int>(std::max(p->n_probes, 1));
  {
    long long nsrc = 0;
    for (int t = 0; t < 6; ++t) nsrc += count_of(p, t);
    L.fpts = cv.take<Fp>(size_t(std::max<long long>(nsrc, 1)));
  }
  L.mons = cv.take<Mon3>(std::max(p->n_monitors, 6));
  L.gsrc = cv.take<long long>(std::max<size_t>(size_t(L.mon_cells), 1));
  L.mring = cv.take<char>(std::max<size_t>(size_t(L.mon_cells) * L.R, 1) * esize);
  L.eacc = cv.take<double>(p->record_energy ? 2 * size_t(std::max(p->n_steps, 1)) : 1);
  long long cw_total = 0;
  if (p->cw_sources)
    for (int t = 0; t < 6; ++t) cw_total += count_of(p, t);
  L.cwv = cv.take<char>(size_t(std::max<long long>(cw_total * L.R, 1)) * esize);
  L.cls = cv.take<unsigned char>(size_t(L.n_cta));
  L.total = cv.bytes();
  return L;
}

static int validate3(const GdnYeeParams* p, const GdnYeePoints* pts, const GdnYeeBuffers* b) {
  if (!p || !pts || !b) GDN_BAD_ARG("null params/points/buffers");
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  if (std::min({nx, ny, nz}) < 3) GDN_BAD_ARG("grid must be at least 3x3x3");
  if (p->npml < 0 || std::min({nx, ny, nz}) <= 2 * p->npml + 2)
    GDN_BAD_ARG("grid %dx%dx%d is too small for CPML thickness %d", nx, ny, nz, p->npml);
  if (p->n_steps < 0 || p->n_freq < 0 || p->n_freq > KMAX || p->n_monitors < 0)
    GDN_BAD_ARG("invalid n_steps / n_freq / n_monitors");
  if ((long long)(nx + 2) * (ny + 2) * (nz + 6) > (1LL << 31))
    GDN_BAD_ARG("grid too large for 32-bit cell ids");
  // Source grids: Jz/probe on Ez edges with margin 1 in i, j (fdtd3d.py:246-255);
  // the other channels anywhere on their own component grid (fdtd3d.py:385-407).
  const int comp_of[7] = {2, 0, 1, 3, 4, 5, 2};
  for (int t = 0; t < 7; ++t) {
    const int n = count_of(p, t);
    const int32_t* a = pts_of(pts, t);
    if (n > 0 && !a) GDN_BAD_ARG("point list %d is null", t);
    int s[3];
    comp_shape(comp_of[t], nx, ny, nz, s);
    const int margin = t == 0 ? 1 : 0;
    for (int m = 0; m < n; ++m) {
      if (t == 6 && pts->probe_comp) {
        const int c = pts->probe_comp[m];
        if (c < 0 || c > 2) GDN_BAD_ARG("probe %d: component %d is not an E component", m, c);
        comp_shape(c, nx, ny, nz, s);
      }
      const int i = a[3 * m], j = a[3 * m + 1], k = a[3 * m + 2];
      if (i < margin || j < margin || k < 0 || i > s[0] - 1 - margin || j > s[1] - 1 - margin ||
          k > s[2] - 1)
        GDN_BAD_ARG("point (%d, %d, %d) of list %d outside its grid", i, j, k, t);
    }
  }
  if (p->has_port) {
    const int i = pts->port[0], j = pts->port[1], k = pts->port[2];
    if (i < 1 || j < 1 || k < 0 || i > nx - 2 || j > ny - 2 || k > nz - 2)
      GDN_BAD_ARG("port (%d, %d, %d) outside the valid Ez range (margin 1)", i, j, k);
    if (p->n_steps > 0 && !b->port_vs) GDN_BAD_ARG("port_vs is null");
    if (p->n_steps > 0 && (!b->out_v || !b->out_i)) GDN_BAD_ARG("port outputs are null");
  }
  if (!b->ca || !b->cb) GDN_BAD_ARG("ca/cb are null");
  for (int a = 0; a < 3; ++a) {
    if (!b->ik_e[a] || !b->ik_h[a]) GDN_BAD_ARG("1/kappa tables are null");
    if (p->npml > 0 && (!b->b_e_lo[a] || !b->c_e_lo[a] || !b->b_e_hi[a] || !b->c_e_hi[a] ||
                        !b->b_h_lo[a] || !b->c_h_lo[a] || !b->b_h_hi[a] || !b->c_h_hi[a]))
      GDN_BAD_ARG("a CPML slab table is null");
  }
  if (!b->ex || !b->ey || !b->ez || !b->hx || !b->hy || !b->hz) GDN_BAD_ARG("field outputs are null");
  if (p->n_probes > 0 && p->n_steps > 0 && !b->out_probe) GDN_BAD_ARG("out_probe is null");
  if (p->record_energy && p->n_steps > 0 && (!b->out_energy || !b->eps))
    GDN_BAD_ARG("energy buffers are null");
  if (p->n_freq > 0 && p->n_steps > 0 && (!b->ph_e || !b->ph_h)) GDN_BAD_ARG("phase tables are null");
  if (p->n_freq > 0 && p->n_monitors == 0)
    for (int c = 0; c < 6; ++c)
      if (!b->dft[c]) GDN_BAD_ARG("full-grid dft output %d is null", c);
  if (p->n_freq > 0 && p->n_monitors > 0) {
    if (!pts->monitors) GDN_BAD_ARG("monitor list is null");
    for (int k = 0; k < p->n_monitors; ++k) {
      const GdnDftMonitor& m = pts->monitors[k];
      if (m.comp < 0 || m.comp > 5) GDN_BAD_ARG("monitor %d: component %d", k, m.comp);
      int s[3];
      comp_shape(m.comp, nx, ny, nz, s);
      for (int a = 0; a < 3; ++a)
        if (m.lo[a] < 0 || m.hi[a] > s[a] || m.hi[a] <= m.lo[a])
          GDN_BAD_ARG("monitor %d: box empty or outside component %d", k, m.comp);
      if (!m.out) GDN_BAD_ARG("monitor %d: output is null", k);
    }
  }
  if (p->cw_sources && (p->n_freq <= 0 || !b->cw_env)) GDN_BAD_ARG("cw_sources needs n_freq and cw_env");
  if (p->n_steps > 0) {
    const void* cur[6] = {b->src_cur, b->jx_cur, b->jy_cur, b->mx_cur, b->my_cur, b->mz_cur};
    const double* w[6] = {b->src_w, b->jx_w, b->jy_w, b->mx_w, b->my_w, b->mz_w};
    for (int t = 0; t < 6; ++t)
      if (count_of(p, t) > 0 && (p->cw_sources ? !w[t] : !cur[t]))
        GDN_BAD_ARG("waveform of point list %d is null", t);
  }
  if ((p->n_src && !b->cb_src) || (p->n_jx && !b->cb_jx) || (p->n_jy && !b->cb_jy))
    GDN_BAD_ARG("source coefficients are null");
  if (p->dt <= 0 || p->dx <= 0 || p->dy <= 0 || p->dz <= 0) GDN_BAD_ARG("dt, dx, dy, dz must be positive");
  return GDN_OK;
}

// Launch with programmatic stream serialisation (see dependent_launch_gate).
template <typename... KArgs, typename... Args>
static void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                       Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Planes per CTA for a step kernel: the CTAs of `cols` (j, k) tile columns
// split the nx planes so that the whole grid is one wave of resident CTAs.
template <typename K>
static int planes_per_cta(K kernel, int nx, int cols, int* ni) {
  int dev = 0, sms = 0, per_sm = 0;
  GDN_TRY_CUDA(cudaGetDevice(&dev));
  GDN_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GDN_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NT, 0));
  const long long slots = (long long)std::max(sms, 1) * std::max(per_sm, 1);
  const long long per_col = std::max<long long>(1, slots / std::max(cols, 1));
  *ni = int(std::max<long long>(1, div_up(nx, per_col)));
  return GDN_OK;
}

template <typename T, typename A>
static void launch_fold3(const Dev3<T>& d, const std::vector<Mon3>& mons, long long max_cells,
                         int cnt, int K, cudaStream_t s) {
  (void)mons;
  (void)max_cells;
  const unsigned dg = unsigned(div_up(d.mon_cells, 256));
  const size_t sm = size_t(4) * cnt * K * sizeof(A);
  if (K <= 4)
    yee_fold<T, A, 4><<<dg, 256, sm, s>>>(d, cnt);
  else if (K <= 8)
    yee_fold<T, A, 8><<<dg, 256, sm, s>>>(d, cnt);
  else
    yee_fold<T, A, KMAX><<<dg, 256, sm, s>>>(d, cnt);
}

template <typename T>
static int run3(const GdnYeeParams* p, const GdnYeePoints* pts, const GdnYeeBuffers* b,
                cudaStream_t stream) {
  int st = validate3(p, pts, b);
  if (st) return st;
  const Layout3 L = make_layout3(p, pts, sizeof(T));
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

  const int nx = p->nx, ny = p->ny, nz = p->nz, N = p->n_steps;
  Dev3<T> d{};
  d.nx = nx; d.ny = ny; d.nz = nz; d.npml = p->npml; d.n_steps = N; d.n_freq = p->n_freq;
  d.R = L.R; d.gj = L.gj; d.gk = L.gk; d.sy = L.sy; d.sz = L.sz; d.vol = L.vol;
  for (int c = 0; c < NC; ++c) d.f[c] = reinterpret_cast<T*>(ws + L.fields) + c * L.vol;
  d.psi = reinterpret_cast<T*>(ws + L.psi);
  d.ca = static_cast<const T*>(b->ca);
  d.cb = static_cast<const T*>(b->cb);
  d.eps = static_cast<const T*>(b->eps);
  for (int a = 0; a < 3; ++a) {
    d.ik_e[a] = static_cast<const T*>(b->ik_e[a]);
    d.ik_h[a] = static_cast<const T*>(b->ik_h[a]);
    d.be_lo[a] = static_cast<const T*>(b->b_e_lo[a]);
    d.ce_lo[a] = static_cast<const T*>(b->c_e_lo[a]);
    d.be_hi[a] = static_cast<const T*>(b->b_e_hi[a]);
    d.ce_hi[a] = static_cast<const T*>(b->c_e_hi[a]);
    d.bh_lo[a] = static_cast<const T*>(b->b_h_lo[a]);
    d.ch_lo[a] = static_cast<const T*>(b->c_h_lo[a]);
    d.bh_hi[a] = static_cast<const T*>(b->b_h_hi[a]);
    d.ch_hi[a] = static_cast<const T*>(b->c_h_hi[a]);
  }
  d.dt_mu = T(b->dt_mu);
  d.inv_d[0] = T(b->inv_dx);
  d.inv_d[1] = T(b->inv_dy);
  d.inv_d[2] = T(b->inv_dz);
  d.dx = T(p->dx); d.dy = T(p->dy); d.dz = T(p->dz);
  d.a_port = T(b->a_port); d.b_port = T(b->b_port); d.c_port = T(b->c_port);
  d.n_src = p->n_src; d.n_jx = p->n_jx; d.n_jy = p->n_jy;
  d.n_mx = p->n_mx; d.n_my = p->n_my; d.n_mz = p->n_mz; d.n_probes = p->n_probes;
  d.has_port = p->has_port;
  d.pi = pts->port[0]; d.pj = pts->port[1]; d.pk = pts->port[2];
  d.port_cta = p->has_port ? (d.pi * L.gj + d.pj / BJ) * L.gk + d.pk / BK : -1;
  d.cb_src = static_cast<const T*>(b->cb_src);
  d.cb_jx = static_cast<const T*>(b->cb_jx);
  d.cb_jy = static_cast<const T*>(b->cb_jy);
  const void* curs[6] = {b->src_cur, b->jx_cur, b->jy_cur, b->mx_cur, b->my_cur, b->mz_cur};
  const double* ws6[6] = {b->src_w, b->jx_w, b->jy_w, b->mx_w, b->my_w, b->mz_w};
  for (int t = 0; t < 6; ++t) {
    d.cur[t] = static_cast<const T*>(curs[t]);
    d.w[t] = reinterpret_cast<const double2*>(ws6[t]);
  }
  d.port_vs = static_cast<const T*>(b->port_vs);
  d.cw = p->cw_sources;
  d.cw_env = b->cw_env;
  d.ph_e = reinterpret_cast<const double2*>(b->ph_e);
  d.ph_h = reinterpret_cast<const double2*>(b->ph_h);
  d.out_probe = static_cast<T*>(b->out_probe);
  d.pcomp = nullptr;
  if (p->n_probes > 0 && pts->probe_comp) {
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.pcomp, pts->probe_comp, size_t(p->n_probes) * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    d.pcomp = reinterpret_cast<const int*>(ws + L.pcomp);
  }
  d.out_v = static_cast<T*>(b->out_v);
  d.out_i = static_cast<T*>(b->out_i);
  d.mring = reinterpret_cast<T*>(ws + L.mring);
  d.mon_cells = L.mon_cells;
  int* step_base = reinterpret_cast<int*>(ws + L.step);
  d.step_base = step_base;
  d.cwv = reinterpret_cast<T*>(ws + L.cwv);
  d.cw_total = 0;
  for (int t = 0; t < 6; ++t) {
    d.cw_off[t] = d.cw_total;
    if (p->cw_sources) d.cw_total += count_of(p, t);
  }

  // Point bins by CTA box (i, j/BJ, k/BK). E sources stay in the step
  // kernel only in boxes that hold probes or the port; every other source
  // point goes to the injection lists.
  auto box_of = [&](int i, int j, int k) { return (i * L.gj + j / BJ) * L.gk + k / BK; };
  std::vector<unsigned char> keep_box(L.n_cta, 0);
  for (int m = 0; m < p->n_probes; ++m)
    keep_box[box_of(pts->probe[3 * m], pts->probe[3 * m + 1], pts->probe[3 * m + 2])] = 1;
  if (p->has_port) keep_box[d.port_cta] = 1;
  auto in_kernel = [&](int t, int c) { return t == 6 || (t <= 2 && keep_box[c]); };
  std::vector<Fp> free_pts[2];
  for (int t = 0; t < 7; ++t) {
    const int n = count_of(p, t);
    const int32_t* a = pts_of(pts, t);
    std::vector<int> off(L.n_cta + 1, 0), cta(n);
    for (int m = 0; m < n; ++m) {
      cta[m] = box_of(a[3 * m], a[3 * m + 1], a[3 * m + 2]);
      if (in_kernel(t, cta[m])) {
        off[cta[m] + 1]++;
      } else {
        const long long cell =
            ((long long)(a[3 * m] + 1) * L.sy + (a[3 * m + 1] + 1)) * L.sz + (a[3 * m + 2] + 1);
        free_pts[t >= 3].push_back(Fp{t, m, cell});
      }
    }
    for (int c = 0; c < L.n_cta; ++c) off[c + 1] += off[c];
    std::vector<Pt3> rec(std::max(n, 1));
    std::vector<int> cur(off.begin(), off.end() - 1);
    for (int m = 0; m < n; ++m)
      if (in_kernel(t, cta[m])) rec[cur[cta[m]]++] = Pt3{m, a[3 * m], a[3 * m + 1], a[3 * m + 2]};
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.off[t], off.data(), off.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    if (n > 0)
      GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.pts[t], rec.data(), size_t(n) * sizeof(Pt3),
                                   cudaMemcpyHostToDevice, stream));
    d.off[t] = reinterpret_cast<const int*>(ws + L.off[t]);
    d.pts[t] = reinterpret_cast<const Pt3*>(ws + L.pts[t]);
  }
  {
    Fp* base = reinterpret_cast<Fp*>(ws + L.fpts);
    for (int side = 0; side < 2; ++side) {
      const size_t nf = free_pts[side].size();
      d.fpts[side] = base + (side ? free_pts[0].size() : 0);
      d.n_fp[side] = (long long)nf;
      if (nf)
        GDN_TRY_CUDA(cudaMemcpyAsync(const_cast<Fp*>(d.fpts[side]), free_pts[side].data(),
                                     nf * sizeof(Fp), cudaMemcpyHostToDevice, stream));
    }
  }

  // Monitors.
  const bool f64acc = p->dft_f64 != 0;
  const size_t csz = f64acc ? sizeof(double2) : sizeof(float2);
  std::vector<Mon3> mons;
  {
    long long off = 0;
    int k = 0;
    for (const auto& bx : mon_boxes3(p, pts)) {
      Mon3 m{};
      m.comp = bx[0];
      m.lo0 = bx[1]; m.lo1 = bx[2]; m.lo2 = bx[3];
      m.s0 = bx[4]; m.s1 = bx[5]; m.s2 = bx[6];
      m.out = p->n_monitors == 0 ? b->dft[k] : pts->monitors[k].out;
      m.count = (long long)m.s0 * m.s1 * m.s2;
      m.off = off;
      off += m.count;
      mons.push_back(m);
      ++k;
    }
  }
  // Ring order: the E-side monitors' cells, then the H-side ones (the fold
  // finds a cell's monitor by binary search over the offsets, so the list
  // is reordered the same way), and the gather table of field offsets.
  {
    std::stable_partition(mons.begin(), mons.end(), [](const Mon3& m) { return m.comp < 3; });
    long long off = 0;
    d.gcells[0] = d.gcells[1] = 0;
    for (Mon3& m : mons) {
      m.off = off;
      off += m.count;
      d.gcells[m.comp >= 3] += m.count;
    }
    std::vector<long long> src(std::max<long long>(L.mon_cells, 1));
    const bool narrow = (long long)NC * L.vol < (1LL << 32);
    for (const Mon3& m : mons) {
      long long r = m.off;
      for (int i = 0; i < m.s0; ++i)
        for (int j = 0; j < m.s1; ++j) {
          const long long row = (long long)m.comp * L.vol +
                                 ((long long)(m.lo0 + i + 1) * L.sy + (m.lo1 + j + 1)) * L.sz +
                                 (m.lo2 + 1);
          for (int k = 0; k < m.s2; ++k) src[r++] = row + k;
        }
    }
    d.gsrc = nullptr;
    d.gsrc64 = nullptr;
    if (narrow) {
      std::vector<unsigned> s32(src.begin(), src.end());
      if (L.mon_cells > 0)
        GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.gsrc, s32.data(), size_t(L.mon_cells) * sizeof(unsigned),
                                     cudaMemcpyHostToDevice, stream));
      d.gsrc = reinterpret_cast<const unsigned*>(ws + L.gsrc);
    } else {
      if (L.mon_cells > 0)
        GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.gsrc, src.data(), size_t(L.mon_cells) * sizeof(long long),
                                     cudaMemcpyHostToDevice, stream));
      d.gsrc64 = reinterpret_cast<const long long*>(ws + L.gsrc);
    }
  }
  d.n_mons = int(mons.size());
  d.mons = reinterpret_cast<const Mon3*>(ws + L.mons);
  // Work flags per plane box: points of the H or E kernel (the port's box
  // counts as E points) and any CPML slab within reach of the box (either
  // field type, a margin of one cell).
  {
    std::vector<unsigned char> cls(L.n_cta, 0);
    for (int t = 0; t < 7; ++t) {
      const int n = count_of(p, t);
      const int32_t* a = pts_of(pts, t);
      for (int m = 0; m < n; ++m) {
        const int c = box_of(a[3 * m], a[3 * m + 1], a[3 * m + 2]);
        if (in_kernel(t, c)) cls[c] |= (t >= 3 && t <= 5) ? F_HPTS : F_EPTS;
      }
    }
    if (p->has_port) cls[d.port_cta] |= F_EPTS;
    const int m = p->npml;
    auto near_slab = [m](int lo, int hi, int n) {  // cells [lo, hi) of an axis of n nodes
      return lo <= m + 1 || hi - 1 >= n - 2 - m;
    };
    for (int i = 0; i < nx; ++i)
      for (int by = 0; by < L.gj; ++by)
        for (int bx = 0; bx < L.gk; ++bx) {
          const bool sl = m > 0 && (near_slab(i, i + 1, nx) ||
                                    near_slab(by * BJ, std::min(ny, (by + 1) * BJ), ny) ||
                                    near_slab(bx * BK, std::min(nz, (bx + 1) * BK), nz));
          if (sl) cls[(i * L.gj + by) * L.gk + bx] |= F_CPML;
        }
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.cls, cls.data(), cls.size(), cudaMemcpyHostToDevice,
                                 stream));
    d.cls = reinterpret_cast<const unsigned char*>(ws + L.cls);
  }
  long long max_cells = 0;
  for (const Mon3& m : mons) {
    max_cells = std::max(max_cells, m.count);
    GDN_TRY_CUDA(cudaMemsetAsync(m.out, 0, size_t(m.count) * p->n_freq * csz, stream));
  }
  if (!mons.empty())
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.mons, mons.data(), mons.size() * sizeof(Mon3),
                                 cudaMemcpyHostToDevice, stream));
  // Start from rest, or from the caller's state blob (fields, then psi).
  const size_t fbytes = size_t(NC) * L.vol * sizeof(T), pbytes = size_t(12) * L.vol * sizeof(T);
  if (b->state_in) {
    const char* si = static_cast<const char*>(b->state_in);
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.fields, si, fbytes, cudaMemcpyDeviceToDevice, stream));
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.psi, si + fbytes, pbytes, cudaMemcpyDeviceToDevice, stream));
    GDN_TRY_CUDA(cudaMemsetAsync(ws + L.step, 0, sizeof(int), stream));
  } else {
    GDN_TRY_CUDA(cudaMemsetAsync(ws + L.fields, 0, L.zero_end - L.fields, stream));
  }
  double* eacc = reinterpret_cast<double*>(ws + L.eacc);
  if (p->record_energy)
    GDN_TRY_CUDA(cudaMemsetAsync(eacc, 0, 2 * size_t(std::max(N, 1)) * sizeof(double), stream));

  const dim3 blk(BK, BJ);
  // Planes per CTA: the fewest that fit every CTA of the grid into one wave
  // of resident CTAs (a partial second wave would idle most SMs).
  int ni_h = 0, ni_e = 0;
  if ((st = planes_per_cta(yee_h<T>, nx, L.gj * L.gk, &ni_h))) return st;
  if ((st = planes_per_cta(yee_e<T>, nx, L.gj * L.gk, &ni_e))) return st;
  const dim3 grd_h(L.gk, L.gj, unsigned(div_up(nx, ni_h)));
  const dim3 grd_e(L.gk, L.gj, unsigned(div_up(nx, ni_e)));
  const int eblocks = int(std::min<long long>(div_up((long long)nx * ny * nz, 256), 148 * 8));
  // Chunk body. With a side stream the ring gathers run beside the step
  // kernels: a gather only reads the field it copies, so the H gather of
  // step t overlaps yee_e of step t and the E gather overlaps yee_h of step
  // t + 1; each field's next writer waits for its gather (events), and the
  // fold waits for the last ones.
  auto enqueue = [&](int cnt, cudaStream_t s, cudaStream_t side, cudaEvent_t* ev) -> uint64_t {
    uint64_t k = 0;
    bool pend_h = false, pend_e = false;  // a gather still reads H / E
    auto gather = [&](int t, int sd, unsigned blocks) {
      if (!side) {
        yee_gather<T><<<blocks, 256, 0, s>>>(d, t, sd);
        return;
      }
      cudaEventRecord(ev[sd], s);
      cudaStreamWaitEvent(side, ev[sd], 0);
      yee_gather<T><<<blocks, 256, 0, side>>>(d, t, sd);
      cudaEventRecord(ev[2 + sd], side);
      (sd ? pend_h : pend_e) = true;
    };
    auto settle = [&](bool& pend, int sd) {  // the field's gather has finished
      if (pend) cudaStreamWaitEvent(s, ev[2 + sd], 0);
      pend = false;
    };
    if (d.cw_total > 0) {
      yee_cw_synth<T><<<unsigned(div_up(d.cw_total, 256)), 256,
                        2 * size_t(cnt) * p->n_freq * sizeof(double2), s>>>(d, cnt);
      ++k;
    }
    const unsigned gb0 = unsigned(div_up(d.gcells[0], 256)), gb1 = unsigned(div_up(d.gcells[1], 256));
    for (int t = 0; t < cnt; ++t) {
      settle(pend_h, 1);
      launch_pdl(yee_h<T>, grd_h, blk, s, d, t, ni_h);
      k += 1;
      if (d.n_fp[1] > 0) {
        launch_pdl(yee_inject<T>, dim3(unsigned(div_up(d.n_fp[1], 256))), dim3(256), s, d, t, 1);
        ++k;
      }
      if (gb1 > 0) {
        gather(t, 1, gb1);
        ++k;
      }
      settle(pend_e, 0);
      launch_pdl(yee_e<T>, grd_e, blk, s, d, t, ni_e);
      k += 1;
      if (d.n_fp[0] > 0) {
        launch_pdl(yee_inject<T>, dim3(unsigned(div_up(d.n_fp[0], 256))), dim3(256), s, d, t, 0);
        ++k;
      }
      if (gb0 > 0) {
        gather(t, 0, gb0);
        ++k;
      }
      if (p->record_energy) {
        yee_energy<T><<<eblocks, 256, 0, s>>>(d, eacc, t);
        ++k;
      }
    }
    settle(pend_h, 1);
    settle(pend_e, 0);
    if (!mons.empty()) {
      if (f64acc)
        launch_fold3<T, double>(d, mons, max_cells, cnt, p->n_freq, s);
      else
        launch_fold3<T, float>(d, mons, max_cells, cnt, p->n_freq, s);
      ++k;
    }
    yee_advance<<<1, 1, 0, s>>>(step_base, cnt);
    return k + 1;
  };
  auto capture = [&](int cnt, cudaGraphExec_t* exec, uint64_t* nodes) -> int {
    cudaStream_t cs = capture_stream();
    if (!cs) GDN_BAD_ARG("no capture stream for this device");
    cudaStream_t side = capture_side_stream();
    cudaEvent_t ev[4] = {};
    bool evs = side != nullptr;
    for (int e = 0; e < 4 && evs; ++e)
      evs = cudaEventCreateWithFlags(&ev[e], cudaEventDisableTiming) == cudaSuccess;
    struct EvGuard {
      cudaEvent_t* e;
      ~EvGuard() {
        for (int q = 0; q < 4; ++q)
          if (e[q]) cudaEventDestroy(e[q]);
      }
    } ev_guard{ev};
    GDN_TRY_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    *nodes = enqueue(cnt, cs, evs ? side : nullptr, ev);
    cudaGraph_t g = nullptr;
    const cudaError_t e1 = cudaStreamEndCapture(cs, &g);
    if (e1 != cudaSuccess) {
      set_error("graph capture failed: %s", cudaGetErrorString(e1));
      return GDN_ERR_CUDA;
    }
    const cudaError_t e2 = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
      set_error("graph instantiate failed: %s", cudaGetErrorString(e2));
      return GDN_ERR_CUDA;
    }
    return GDN_OK;
  };
  const int Tc = L.R, full = N / Tc, rem = N % Tc;
  cudaGraphExec_t g_full = nullptr, g_rem = nullptr;
  uint64_t k_full = 0, k_rem = 0;
  if (full > 0 && (st = capture(Tc, &g_full, &k_full))) return st;
  if (rem > 0 && (st = capture(rem, &g_rem, &k_rem))) {
    if (g_full) cudaGraphExecDestroy(g_full);
    return st;
  }
  cudaError_t le = cudaSuccess;
  LoopTimer timer(stream, double(p->nx) * p->ny * p->nz * p->n_steps, p->n_steps);
  for (int c = 0; c < full && le == cudaSuccess; ++c) le = cudaGraphLaunch(g_full, stream);
  if (rem > 0 && le == cudaSuccess) le = cudaGraphLaunch(g_rem, stream);
  timer.stop(le == cudaSuccess);
  if (g_full) cudaGraphExecDestroy(g_full);
  if (g_rem) cudaGraphExecDestroy(g_rem);
  if (le != cudaSuccess) {
    set_error("graph launch failed: %s", cudaGetErrorString(le));
    return GDN_ERR_CUDA;
  }
  count_launches(uint64_t(full) * k_full + k_rem);

  yee_copy_out<T><<<eblocks, 256, 0, stream>>>(
      d, static_cast<T*>(b->ex), static_cast<T*>(b->ey), static_cast<T*>(b->ez),
      static_cast<T*>(b->hx), static_cast<T*>(b->hy), static_cast<T*>(b->hz));
  for (const Mon3& m : mons) {
    const long long cnt = m.count * p->n_freq;
    const int blocks = int(std::min<long long>(div_up(cnt, 256), 148 * 8));
    if (f64acc)
      yee_dft_scale<double2><<<blocks, 256, 0, stream>>>(static_cast<double2*>(m.out), cnt, p->dt);
    else
      yee_dft_scale<float2><<<blocks, 256, 0, stream>>>(static_cast<float2*>(m.out), cnt, p->dt);
  }
  if (b->state_out) {
    char* so = static_cast<char*>(b->state_out);
    GDN_TRY_CUDA(cudaMemcpyAsync(so, ws + L.fields, fbytes, cudaMemcpyDeviceToDevice, stream));
    GDN_TRY_CUDA(cudaMemcpyAsync(so + fbytes, ws + L.psi, pbytes, cudaMemcpyDeviceToDevice, stream));
  }
  if (p->record_energy && N > 0)
    yee_energy_finish<T><<<unsigned(div_up(N, 256)), 256, 0, stream>>>(
        eacc, static_cast<T*>(b->out_energy), N, p->dx * p->dy * p->dz, p->mu0);
  count_launches(1 + mons.size() + (p->record_energy && N > 0 ? 1 : 0));
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

}  // namespace yee3d
}  // namespace gdn

extern "C" int gdn_yee_workspace_size(const GdnYeeParams* p, const GdnYeePoints* pts, int f64,
                                      size_t* bytes) {
  if (!p || !bytes) {
    gdn::set_error("null argument");
    return GDN_ERR_BAD_ARG;
  }
  if (std::min({p->nx, p->ny, p->nz}) < 3 || p->npml < 0) {
    gdn::set_error("invalid grid");
    return GDN_ERR_BAD_ARG;
  }
  if (p->n_freq > 0 && p->n_monitors > 0 && (!pts || !pts->monitors)) {
    gdn::set_error("monitor list is null");
    return GDN_ERR_BAD_ARG;
  }
  *bytes = gdn::yee3d::make_layout3(p, pts, f64 ? sizeof(double) : sizeof(float)).total;
  return GDN_OK;
}

extern "C" int gdn_yee_state_size(const GdnYeeParams* p, int f64, size_t* bytes) {
  if (!p || !bytes) {
    gdn::set_error("null argument");
    return GDN_ERR_BAD_ARG;
  }
  if (std::min({p->nx, p->ny, p->nz}) < 3) {
    gdn::set_error("invalid grid");
    return GDN_ERR_BAD_ARG;
  }
  const long long sz = gdn::div_up(p->nz + 2, 4) * 4;
  const long long vol = (long long)(p->nx + 2) * (p->ny + 2) * sz;
  *bytes = size_t(gdn::yee3d::NC + 12) * size_t(vol) * (f64 ? sizeof(double) : sizeof(float));
  return GDN_OK;
}

extern "C" int gdn_yee_run_f32(const GdnYeeParams* p, const GdnYeePoints* pts,
                               const GdnYeeBuffers* b, void* stream) {
  return gdn::yee3d::run3<float>(p, pts, b, static_cast<cudaStream_t>(stream));
}

extern "C" int gdn_yee_run_f64(const GdnYeeParams* p, const GdnYeePoints* pts,
                               const GdnYeeBuffers* b, void* stream) {
  return gdn::yee3d::run3<double>(p, pts, b, static_cast<cudaStream_t>(stream));
}
