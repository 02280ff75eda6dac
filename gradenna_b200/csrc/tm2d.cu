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
//   * Temporal blocking. One launch advances TB time steps. A CTA owns a
//     TI x TJ tile of cells and stages Ez, Hx, Hy, ca and cb for the tile plus
//     a halo (TB rows, HJ >= TB columns) in shared memory with 16-byte
//     cp.async copies, then runs the TB sub-steps entirely in shared memory:
//     each sub-step's H and E sweeps also cover the halo (redundantly with the
//     neighbours), whose valid part shrinks by one cell per sub-step, so the
//     owned tile stays exact. Global traffic and launches drop by TB.
//   * Field state is a ping-pong pair of padded planes (ghost rows/columns
//     stay zero: they are also the PEC ring); launch k reads pair k&1 and
//     writes pair (k+1)&1, so halo reads never race with owners' writes.
//   * Two tile classes run as two concurrent launches per block: interior
//     tiles (no CPML, no PEC ring: five staged planes, branch-free vector
//     sweeps) and general tiles, which also stage the four CPML psi planes
//     (ezx, ezy, hyx, hxy: padded planes, zero outside the slabs, ping-pong
//     by launch parity like the fields) and use per-row/column coefficient
//     and mask tables so their sweeps are branch-free too.
//   * Point work (sources, ports, probes, magnetic currents) is binned on the
//     host into per-tile lists that include the halo; injections are applied
//     to every copy of a cell, records (V, I, probes) only by the owner.
//   * The running DFT reads a compact MONITOR RING: every sub-step the owner
//     writes the monitored cells' values (only those) into ring slot n % R;
//     once per R steps one fold kernel adds sum_t ph[t,k] x_t to the
//     accumulators, so accumulator read-modify-write traffic drops by R.
//   * One chunk of R steps (R/TB step launches + fold + counter advance) is
//     captured once as a CUDA graph and replayed; kernels read the absolute
//     step index from a device counter.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace gdn {
namespace tm2d {

constexpr int PADJ = 32;  // ghost columns on each side of a plane (>= HJ)
constexpr int PADI = 8;   // ghost rows above and below a plane (>= TB)
constexpr int HJ = 4;     // column halo in shared memory (16 bytes of f32)
constexpr int KMAX = 16;  // most DFT frequencies per run
constexpr int MAXP = 64;  // most port records in one tile

// Tile configurations (TB sub-steps, TI x TJ owned cells, NT threads).
struct Cfg {
  int tb, ti, tj, nt;
};
// Per field type five shapes: three with TB = 4 (largest first) and two
// with TB = 2. pick_cfg chooses a TB = 4 one from the grid size;
// GDN_TM_TILE=0..4 or the batched entry point's `cfg` argument (set by the
// autotuner) forces any. The one-step shape serves runs that record the
// energy every step.
constexpr int NCFG = 5;
constexpr Cfg kCfgF32[NCFG] = {
    {4, 64, 64, 512}, {4, 32, 64, 256}, {4, 16, 32, 128}, {2, 64, 64, 512}, {2, 32, 64, 256}};
constexpr Cfg kCfgF64[NCFG] = {
    {4, 28, 64, 512}, {4, 16, 64, 256}, {4, 16, 32, 128}, {2, 28, 64, 512}, {2, 16, 64, 256}};
constexpr Cfg kCfgStep{1, 16, 64, 256};  // one step per launch (energy records)

struct Pt {
  int m, i, j, owner;  // point index, cell, 1 if this tile owns the cell
};

// A DFT monitor resolved against the grid: box [lo0, lo0+h) x [lo1, lo1+w)
// of component comp, stored at `off` in every monitor-ring slot.
struct MonD {
  int comp, lo0, lo1, h, w, pad;
  long long count, off;
  void* out;
};

// One monitor's part inside one tile: cells [a0, a1) x [b0, b1) of
// component comp, written to ring index base + i * w + j. Binned per tile on
// the host so a tile touches only the monitors that cross it.
struct MonW {
  int a0, a1, b0, b1, comp, w;
  long long base;
};
constexpr int MAXW = 16;  // per-tile monitor parts staged in shared memory
constexpr int MAXF = 64;  // monitors whose offsets the fold stages in shared memory

// Row-march work item (one warp): owned rows [i0, i0 + rows) and owned
// columns [j0, j0 + owned_cols), its point entries [pb, pe) in MPt order and
// its monitor parts [mb, me).
struct MTask {
  int i0, j0, rows, cls, pb, pe, mb, me;
};

// A row-march point entry: cell (i, j), point index m, tag = type (bits 0-2,
// march::P_*) | 8 if the warp owns the cell (records are written by owners).
struct MPt {
  int i, j, m, tag;
};

template <typename T>
struct Dev {
  int nx, ny, ld, npml, n_steps, n_freq, R, tiles_x;
  long long plane;    // elements per padded plane
  T* state[2];        // ping-pong field slots, 3 planes each (ez, hx, hy)
  T* mring;           // monitor ring: R slots x mon_cells
  long long mon_cells;
  int n_mons;
  const MonD* mons;
  const int* mw_off;  // per-tile CSR over mw
  const MonW* mw;
  const T *ca, *cb, *eps;  // ca/cb padded planes; eps caller (nx, ny)
  const T *ikx_e, *iky_e, *ikx_h, *iky_h;
  const T *b_ezx_lo, *c_ezx_lo, *b_ezx_hi, *c_ezx_hi;
  const T *b_ezy_lo, *c_ezy_lo, *b_ezy_hi, *c_ezy_hi;
  const T *b_hyx_lo, *c_hyx_lo, *b_hyx_hi, *c_hyx_hi;
  const T *b_hxy_lo, *c_hxy_lo, *b_hxy_hi, *c_hxy_hi;
  // CPML psi as padded planes (zero outside the slabs), by launch parity:
  // 4 consecutive planes ezx, ezy, hyx, hxy per parity.
  T* psi[2];
  T dt_mu, inv_dx, inv_dy, dx, dy, dz;
  int n_src, n_ports, n_mx, n_my, n_probes;
  const int *src_off, *port_off, *mx_off, *my_off, *probe_off;
  const Pt *src_pts, *port_pts, *mx_pts, *my_pts, *probe_pts;
  const T *cb_src, *src_cur, *cb_vs, *port_vs, *mx_cur, *my_cur;
  int cw;
  const double* cw_env;
  const double2 *src_w, *mx_w, *my_w, *ph_e, *ph_h;
  T *out_probe, *out_v, *out_i;
  const int* step_base;
  const MPt* mpts;  // row-march point entries (sorted by warp, then row, then type)
};

// Offset of field cell (i, j) in a padded plane.
__device__ __host__ __forceinline__ long long cell_at(int ld, int i, int j) {
  return (long long)(i + PADI) * ld + (j + PADJ);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Value of a point source waveform at step n: tabulated, or synthesised from
// CW phasor weights, J(n) = env[n] Re(sum_k W_k conj(ph[n,k])).
template <typename T>
__device__ __forceinline__ T point_value(const Dev<T>& d, const T* cur, const double2* w,
                                         const double2* ph, int n_pts, int m, int n) {
  if (!d.cw) return cur[(long long)n * n_pts + m];
  double s = 0.0;
  for (int k = 0; k < d.n_freq; ++k) {
    const double2 a = w[(long long)m * d.n_freq + k];
    const double2 p = ph[(long long)n * d.n_freq + k];
    s += a.x * p.x + a.y * p.y;
  }
  return T(d.cw_env[n] * s);
}

// ---------------------------------------------------------------------------
// Point work of one sub-step on the staged region (fdtd2d.py:419-451, 461).
// ---------------------------------------------------------------------------
struct TileLists {
  int mb, me, yb, ye, sb, se, pb, pe, qb, qe;
};

// Point-source values of a launch are staged once in shared memory (sVal):
// item (k * TB + s) is the k-th record of the tile's Jz list at sub-step s,
// then the Mx list, then the My list; items past MAXV are computed in place.
template <typename T>
struct Vals {
  static constexpr int MAXV = 4096 / int(sizeof(T));
};

template <typename T>
__device__ __forceinline__ T src_term(const Dev<T>& d, int m, int n) {
  return d.cb_src[m] * point_value(d, d.src_cur, d.src_w, d.ph_e, d.n_src, m, n);
}
template <typename T>
__device__ __forceinline__ T mx_term(const Dev<T>& d, int m, int n) {
  return d.dt_mu * point_value(d, d.mx_cur, d.mx_w, d.ph_h, d.n_mx, m, n);
}
template <typename T>
__device__ __forceinline__ T my_term(const Dev<T>& d, int m, int n) {
  return d.dt_mu * point_value(d, d.my_cur, d.my_w, d.ph_h, d.n_my, m, n);
}

template <typename T, int TB, int NT>
__device__ __forceinline__ void stage_values(const Dev<T>& d, const TileLists& L, T* sVal,
                                             int n0, int nsub, int tid) {
  constexpr int MAXV = Vals<T>::MAXV;
  const int nj = (L.se - L.sb) * TB, nxm = (L.me - L.mb) * TB, nym = (L.ye - L.yb) * TB;
  const int tot = min(nj + nxm + nym, MAXV);
  for (int q = tid; q < tot; q += NT) {
    const int s = q % TB;
    if (s >= nsub) continue;
    if (q < nj) {
      sVal[q] = src_term(d, d.src_pts[L.sb + q / TB].m, n0 + s);
    } else if (q < nj + nxm) {
      sVal[q] = mx_term(d, d.mx_pts[L.mb + (q - nj) / TB].m, n0 + s);
    } else {
      sVal[q] = my_term(d, d.my_pts[L.yb + (q - nj - nxm) / TB].m, n0 + s);
    }
  }
}

template <typename T, int TB, int EW, int NT>
__device__ __forceinline__ void apply_magnetic(const Dev<T>& d, const TileLists& L, T* sHx,
                                               T* sHy, const T* sVal, int ie, int je, int n,
                                               int s, int tid) {
  constexpr int MAXV = Vals<T>::MAXV;
  const int nj = (L.se - L.sb) * TB, nxm = (L.me - L.mb) * TB;
  for (int q = L.mb + tid; q < L.me; q += NT) {
    const Pt pt = d.mx_pts[q];
    const int v = nj + (q - L.mb) * TB + s;
    atomicAdd(&sHx[(pt.i - ie) * EW + (pt.j - je)], -(v < MAXV ? sVal[v] : mx_term(d, pt.m, n)));
  }
  for (int q = L.yb + tid; q < L.ye; q += NT) {
    const Pt pt = d.my_pts[q];
    const int v = nj + nxm + (q - L.yb) * TB + s;
    atomicAdd(&sHy[(pt.i - ie) * EW + (pt.j - je)], -(v < MAXV ? sVal[v] : my_term(d, pt.m, n)));
  }
}

// Monitored cells of the tile for the Ez monitors (want_e) or the Hx/Hy
// monitors (!want_e) into ring slot n % R: only the monitor parts binned to
// this tile; one warp per row, lanes along it.
template <typename T, int EW, int NT>
__device__ __forceinline__ void write_ring(const Dev<T>& d, const MonW* sMW, int wb, int nw,
                                           bool want_e, const T* sEz, const T* sHx,
                                           const T* sHy, int ie, int je, int n, int tid) {
  constexpr int NW = NT / 32;
  const int warp = tid >> 5, lane = tid & 31;
  T* slot = d.mring + (long long)(n % d.R) * d.mon_cells;
  auto part = [&](const MonW& e) {
    if ((e.comp == 0) != want_e) return;
    const T* f = (e.comp == 0 ? sEz : (e.comp == 1 ? sHx : sHy)) - je;
    T* o = slot + e.base;
    for (int i = e.a0 + warp; i < e.a1; i += NW) {
      const T* fr = f + (i - ie) * EW;
      T* orow = o + (long long)i * e.w;
      for (int j = e.b0 + lane; j < e.b1; j += 32) orow[j] = fr[j];
    }
  };
  const int ns = min(nw, MAXW);
  for (int q = 0; q < ns; ++q) part(sMW[q]);
  for (int q = MAXW; q < nw; ++q) part(d.mw[wb + q]);
}

// Per-row / per-column CPML coefficients and validity masks of a general
// tile, so its sweeps are branch-free: outside the slabs b = c = 0 and
// 1/kappa = 1, which reproduces the plain update exactly (psi stays 0).
template <typename T, int EH, int EW>
struct Coef {
  T rb_h[EH], rc_h[EH], rk_h[EH], rb_e[EH], rc_e[EH], rk_e[EH];  // hyx, ezx (by row)
  T cb_h[EW], cc_h[EW], ck_h[EW], cb_e[EW], cc_e[EW], ck_e[EW];  // hxy, ezy (by column)
  unsigned char r_hx[EH], r_hy[EH], r_e[EH], c_hx[EW], c_hy[EW], c_e[EW];
  // psi in use: rows inside an x slab (hyx, ezx) and 16-byte column groups
  // touching a y slab (hxy, ezy). Elsewhere the psi recursion is identically
  // zero (b = c = 0, 1/kappa = 1) and the sweeps skip it.
  unsigned char x_h[EH], x_e[EH], y_h[EW / (16 / sizeof(T))], y_e[EW / (16 / sizeof(T))];
};

template <typename T, int EH, int EW, int NT>
__device__ void fill_coef(const Dev<T>& d, Coef<T, EH, EW>& k, int ie, int je, int tid) {
  const int nx = d.nx, ny = d.ny, m = d.npml;
  for (int r = tid; r < EH; r += NT) {
    const int i = ie + r;
    T b = 0, c = 0, kk = 1;
    if (i >= 0 && i < nx - 1) {
      if (i < m) {
        b = d.b_hyx_lo[i]; c = d.c_hyx_lo[i]; kk = d.ikx_h[i];
      } else if (i >= nx - 1 - m) {
        b = d.b_hyx_hi[i - (nx - 1 - m)]; c = d.c_hyx_hi[i - (nx - 1 - m)]; kk = d.ikx_h[i];
      }
    }
    k.rb_h[r] = b; k.rc_h[r] = c; k.rk_h[r] = kk;
    const int a = i - 1, ni = nx - 2;
    b = 0; c = 0; kk = 1;
    if (a >= 0 && a < ni) {
      if (a < m) {
        b = d.b_ezx_lo[a]; c = d.c_ezx_lo[a]; kk = d.ikx_e[a];
      } else if (a >= ni - m) {
        b = d.b_ezx_hi[a - (ni - m)]; c = d.c_ezx_hi[a - (ni - m)]; kk = d.ikx_e[a];
      }
    }
    k.rb_e[r] = b; k.rc_e[r] = c; k.rk_e[r] = kk;
    k.r_hx[r] = i >= 0 && i < nx;
    k.r_hy[r] = i >= 0 && i < nx - 1;
    k.r_e[r] = i >= 1 && i <= nx - 2;
    k.x_h[r] = i >= 0 && i < nx - 1 && (i < m || i >= nx - 1 - m);
    k.x_e[r] = a >= 0 && a < ni && (a < m || a >= ni - m);
  }
  constexpr int V = 16 / sizeof(T);
  for (int g = tid; g < EW / V; g += NT) {
    bool h = false, e = false;
    for (int u = 0; u < V; ++u) {
      const int j = je + g * V + u, bb = j - 1;
      h = h || (j >= 0 && j < ny - 1 && (j < m || j >= ny - 1 - m));
      e = e || (bb >= 0 && bb < ny - 2 && (bb < m || bb >= ny - 2 - m));
    }
    k.y_h[g] = h;
    k.y_e[g] = e;
  }
  for (int cidx = tid; cidx < EW; cidx += NT) {
    const int j = je + cidx;
    T b = 0, c = 0, kk = 1;
    if (j >= 0 && j < ny - 1) {
      if (j < m) {
        b = d.b_hxy_lo[j]; c = d.c_hxy_lo[j]; kk = d.iky_h[j];
      } else if (j >= ny - 1 - m) {
        b = d.b_hxy_hi[j - (ny - 1 - m)]; c = d.c_hxy_hi[j - (ny - 1 - m)]; kk = d.iky_h[j];
      }
    }
    k.cb_h[cidx] = b; k.cc_h[cidx] = c; k.ck_h[cidx] = kk;
    const int bb = j - 1, nj = ny - 2;
    b = 0; c = 0; kk = 1;
    if (bb >= 0 && bb < nj) {
      if (bb < m) {
        b = d.b_ezy_lo[bb]; c = d.c_ezy_lo[bb]; kk = d.iky_e[bb];
      } else if (bb >= nj - m) {
        b = d.b_ezy_hi[bb - (nj - m)]; c = d.c_ezy_hi[bb - (nj - m)]; kk = d.iky_e[bb];
      }
    }
    k.cb_e[cidx] = b; k.cc_e[cidx] = c; k.ck_e[cidx] = kk;
    k.c_hx[cidx] = j >= 0 && j < ny - 1;
    k.c_hy[cidx] = j >= 0 && j < ny;
    k.c_e[cidx] = j >= 1 && j <= ny - 2;
  }
}

// The row-march kernel (defined in this namespace).
#include "tm2d_march.cuh"

template <typename T>
__device__ __forceinline__ void ld16(T* dst, const T* src) {
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
}
template <typename T>
__device__ __forceinline__ void st16(T* dst, const T* src) {
  *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
}

// ---------------------------------------------------------------------------
// TB fused time steps on one tile + halo (fdtd2d.py:412-464 per sub-step).
// GEN = true: tiles that touch the CPML slabs or the PEC ring; psi of the
// extended region lives in shared memory and per-row/column coefficients and
// masks make the sweeps branch-free. GEN = false: interior tiles, no psi and
// no masks. Both sweep 16-byte vectors of cells along a row.
// ---------------------------------------------------------------------------
template <typename T, int TB, int TI, int TJ, int NT, bool GEN>
__device__ __forceinline__ void tb_body(const Dev<T>& d, const int tile, int sub0, int nsub) {
  constexpr int EH = TI + 2 * TB;  // extended rows
  constexpr int EW = TJ + 2 * HJ;  // extended columns
  constexpr int EC = EH * EW;
  constexpr int V = 16 / sizeof(T);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sEz = reinterpret_cast<T*>(smem_raw);
  T* sHx = sEz + EC;
  T* sHy = sHx + EC;
  T* sCa = sHy + EC;
  T* sCb = sCa + EC;
  T* sPsi = sCb + EC;  // GEN only: ezx, ezy, hyx, hxy
  __shared__ T sEb[MAXP];       // Ez^n at owned port records
  __shared__ T sPv[MAXP * TB];  // cb_vs * Vs of the tile's port records per sub-step
  __shared__ Coef<T, GEN ? EH : 1, GEN ? EW : 1> K;

  const int n0 = *d.step_base + sub0;
  const int par = (n0 / TB) & 1;
  const int nx = d.nx, ny = d.ny, ld = d.ld, npml = d.npml;
  const int ty = tile / d.tiles_x, tx = tile - ty * d.tiles_x;
  const int i0 = ty * TI, j0 = tx * TJ;
  const int ie = i0 - TB, je = j0 - HJ;  // global cell of extended (0, 0)
  const int tid = threadIdx.x;
  const T* src = d.state[par];
  T* dst = d.state[par ^ 1];

  // ---- stage the extended region (16-byte async copies) ----
  constexpr int CW = EW / V;
  for (int q = tid; q < EH * CW; q += NT) {
    const int r = q / CW, c = (q - r * CW) * V;
    const long long g = cell_at(ld, ie + r, je + c);
    cp_async16(sEz + r * EW + c, src + g);
    cp_async16(sHx + r * EW + c, src + d.plane + g);
    cp_async16(sHy + r * EW + c, src + 2 * d.plane + g);
    cp_async16(sCa + r * EW + c, d.ca + g);
    cp_async16(sCb + r * EW + c, d.cb + g);
  }
  if constexpr (GEN) {
    const T* gp = d.psi[par];
    for (int q = tid; q < EH * CW; q += NT) {
      const int r = q / CW, c = (q - r * CW) * V;
      const long long g = cell_at(ld, ie + r, je + c);
      for (int t = 0; t < 4; ++t) cp_async16(sPsi + t * EC + r * EW + c, gp + t * d.plane + g);
    }
    fill_coef<T, EH, EW, NT>(d, K, ie, je, tid);
  }
  TileLists tl;
  tl.mb = d.mx_off[tile]; tl.me = d.mx_off[tile + 1];
  tl.yb = d.my_off[tile]; tl.ye = d.my_off[tile + 1];
  tl.sb = d.src_off[tile]; tl.se = d.src_off[tile + 1];
  tl.pb = d.port_off[tile]; tl.pe = d.port_off[tile + 1];
  tl.qb = d.probe_off[tile]; tl.qe = d.probe_off[tile + 1];
  for (int q = tid; q < (tl.pe - tl.pb) * nsub; q += NT) {
    const int k = q / nsub, s = q - k * nsub;
    const int m = d.port_pts[tl.pb + k].m;
    sPv[k * TB + s] = d.cb_vs[m] * d.port_vs[(long long)(n0 + s) * d.n_ports + m];
  }
  __shared__ MonW sMW[MAXW];
  int wb = 0, nw = 0;
  if (d.n_mons > 0) {
    wb = d.mw_off[tile];
    nw = d.mw_off[tile + 1] - wb;
    for (int q = tid; q < min(nw, MAXW); q += NT) sMW[q] = d.mw[wb + q];
  }
  __shared__ T sVal[Vals<T>::MAXV];
  stage_values<T, TB, NT>(d, tl, sVal, n0, nsub, tid);
  cp_async_wait_all();
  __syncthreads();
  const T dt_mu = d.dt_mu, inv_dx = d.inv_dx, inv_dy = d.inv_dy;

  for (int s = 0; s < nsub; ++s) {
    const int n = n0 + s;
    // ---- H sweep (fdtd2d.py:416-428) over the extended region ----
    // The last element's right neighbour and the last row's lower neighbour
    // read past the row: garbage that, like every halo value, only reaches
    // cells outside the owned tile within TB sub-steps.
    for (int q = tid * V; q < EC; q += NT * V) {
      T e[V + 1], el[V], hx[V], hy[V];
      ld16(e, sEz + q);
      e[V] = sEz[q + V];
      ld16(el, sEz + q + EW);
      ld16(hx, sHx + q);
      ld16(hy, sHy + q);
      if constexpr (GEN) {
        const int r = q / EW, c = q - r * EW;
        const bool sy = K.y_h[c / V], sx = K.x_h[r];
        T pxy[V], pyx[V];
        if (sy) ld16(pxy, sPsi + 3 * EC + q);
        if (sx) ld16(pyx, sPsi + 2 * EC + q);
        const T rb = K.rb_h[r], rc = K.rc_h[r], rk = K.rk_h[r];
        const bool rhx = K.r_hx[r], rhy = K.r_hy[r];
#pragma unroll
        for (int k = 0; k < V; ++k) {
          const T dy_ = (e[k + 1] - e[k]) * inv_dy;
          T thx = dy_;
          if (sy) {
            pxy[k] = K.cb_h[c + k] * pxy[k] + K.cc_h[c + k] * dy_;
            thx = dy_ * K.ck_h[c + k] + pxy[k];
          }
          if (rhx && K.c_hx[c + k]) hx[k] -= dt_mu * thx;
          const T dx_ = (el[k] - e[k]) * inv_dx;
          T thy = dx_;
          if (sx) {
            pyx[k] = rb * pyx[k] + rc * dx_;
            thy = dx_ * rk + pyx[k];
          }
          if (rhy && K.c_hy[c + k]) hy[k] += dt_mu * thy;
        }
        if (sy) st16(sPsi + 3 * EC + q, pxy);
        if (sx) st16(sPsi + 2 * EC + q, pyx);
      } else {
#pragma unroll
        for (int k = 0; k < V; ++k) {
          hx[k] -= dt_mu * ((e[k + 1] - e[k]) * inv_dy);
          hy[k] += dt_mu * ((el[k] - e[k]) * inv_dx);
        }
      }
      st16(sHx + q, hx);
      st16(sHy + q, hy);
    }
    // Ez monitors of the previous sub-step (Ez is not written in this phase).
    if (nw > 0 && s > 0) write_ring<T, EW, NT>(d, sMW, wb, nw, true, sEz, sHx, sHy, ie, je, n - 1, tid);
    __syncthreads();
    if (tl.mb < tl.me || tl.yb < tl.ye) {
      apply_magnetic<T, TB, EW, NT>(d, tl, sHx, sHy, sVal, ie, je, n, s, tid);
      __syncthreads();
    }
    // Port current on H^{n+1/2} and the Ez^n snapshot (fdtd2d.py:430-436).
    if (tl.pb < tl.pe) {
      for (int q = tl.pb + tid; q < tl.pe; q += NT) {
        const Pt pt = d.port_pts[q];
        if (!pt.owner) continue;
        const int l = (pt.i - ie) * EW + (pt.j - je);
        sEb[q - tl.pb] = sEz[l];
        d.out_i[(long long)n * d.n_ports + pt.m] =
            (sHy[l] - sHy[l - EW]) * d.dy - (sHx[l] - sHx[l - 1]) * d.dx;
      }
      __syncthreads();
    }
    // ---- E sweep (fdtd2d.py:438-443), in place ----
    for (int q = tid * V; q < EC; q += NT * V) {
      T e[V], ca[V], cb[V], hx[V + 1], hy[V], hu[V];
      ld16(e, sEz + q);
      ld16(ca, sCa + q);
      ld16(cb, sCb + q);
      hx[0] = q > 0 ? sHx[q - 1] : T(0);
      ld16(hx + 1, sHx + q);
      ld16(hy, sHy + q);
      ld16(hu, sHy + (q >= EW ? q - EW : q));
      if constexpr (GEN) {
        const int r = q / EW, c = q - r * EW;
        const bool sx = K.x_e[r], sy = K.y_e[c / V];
        T px[V], py[V];
        if (sx) ld16(px, sPsi + q);
        if (sy) ld16(py, sPsi + EC + q);
        const T rb = K.rb_e[r], rc = K.rc_e[r], rk = K.rk_e[r];
        const bool re = K.r_e[r];
#pragma unroll
        for (int k = 0; k < V; ++k) {
          const T dhy_dx = (hy[k] - hu[k]) * inv_dx;
          const T dhx_dy = (hx[k + 1] - hx[k]) * inv_dy;
          T tx_ = dhy_dx, ty_ = dhx_dy;
          if (sx) {
            px[k] = rb * px[k] + rc * dhy_dx;
            tx_ = dhy_dx * rk + px[k];
          }
          if (sy) {
            py[k] = K.cb_e[c + k] * py[k] + K.cc_e[c + k] * dhx_dy;
            ty_ = dhx_dy * K.ck_e[c + k] + py[k];
          }
          if (re && K.c_e[c + k]) e[k] = ca[k] * e[k] + cb[k] * (tx_ - ty_);
        }
        if (sx) st16(sPsi + q, px);
        if (sy) st16(sPsi + EC + q, py);
      } else {
#pragma unroll
        for (int k = 0; k < V; ++k)
          e[k] = ca[k] * e[k] + cb[k] * ((hy[k] - hu[k]) * inv_dx - (hx[k + 1] - hx[k]) * inv_dy);
      }
      st16(sEz + q, e);
    }
    // H monitors of this sub-step (H is final and only read in this phase).
    if (nw > 0) write_ring<T, EW, NT>(d, sMW, wb, nw, false, sEz, sHx, sHy, ie, je, n, tid);
    __syncthreads();
    // Jz line sources on every copy: Ez -= cb_src J (fdtd2d.py:444).
    if (tl.sb < tl.se) {
      for (int q = tl.sb + tid; q < tl.se; q += NT) {
        const Pt pt = d.src_pts[q];
        const int v = (q - tl.sb) * TB + s;
        atomicAdd(&sEz[(pt.i - ie) * EW + (pt.j - je)],
                  -(v < Vals<T>::MAXV ? sVal[v] : src_term(d, pt.m, n)));
      }
      __syncthreads();
    }
    // RVS ports in port order: every injection, then V for owned records.
    if (tl.pb < tl.pe) {
      if (tid == 0) {
        for (int q = tl.pb; q < tl.pe; ++q) {
          const Pt pt = d.port_pts[q];
          sEz[(pt.i - ie) * EW + (pt.j - je)] += -sPv[(q - tl.pb) * TB + s];
        }
        for (int q = tl.pb; q < tl.pe; ++q) {
          const Pt pt = d.port_pts[q];
          if (pt.owner)
            d.out_v[(long long)n * d.n_ports + pt.m] =
                T(-0.5) * d.dz * (sEb[q - tl.pb] + sEz[(pt.i - ie) * EW + (pt.j - je)]);
        }
      }
      __syncthreads();
    }
    for (int q = tl.qb + tid; q < tl.qe; q += NT) {
      const Pt pt = d.probe_pts[q];
      d.out_probe[(long long)n * d.n_probes + pt.m] = sEz[(pt.i - ie) * EW + (pt.j - je)];
    }
  }
  // Ez monitors of the last sub-step, in the same read-only phase as the
  // write-back below.
  if (nw > 0 && nsub > 0)
    write_ring<T, EW, NT>(d, sMW, wb, nw, true, sEz, sHx, sHy, ie, je, n0 + nsub - 1, tid);

  // ---- owned fields to the other state slot; owned psi back to the slabs ----
  constexpr int TV = TJ / V;
  for (int q = tid; q < TI * TV; q += NT) {
    const int r = q / TV, c = (q - r * TV) * V;
    const long long g = cell_at(ld, i0 + r, j0 + c);
    const int l = (r + TB) * EW + (c + HJ);
    st16(dst + g, sEz + l);
    st16(dst + d.plane + g, sHx + l);
    st16(dst + 2 * d.plane + g, sHy + l);
  }
  if constexpr (GEN) {
    T* gp = d.psi[par ^ 1];
    for (int q = tid; q < TI * TV; q += NT) {
      const int r = q / TV, c = (q - r * TV) * V;
      const long long g = cell_at(ld, i0 + r, j0 + c);
      const int l = (r + TB) * EW + (c + HJ);
      for (int t = 0; t < 4; ++t) st16(gp + t * d.plane + g, sPsi + t * EC + l);
    }
  }
}

template <typename T, int TB, int TI, int TJ, int NT, bool GEN>
__global__ void __launch_bounds__(NT) tm_tb(Dev<T> d, const int* tiles, int sub0, int nsub) {
  tb_body<T, TB, TI, TJ, NT, GEN>(d, tiles[blockIdx.x], sub0, nsub);
}

// Batched form: CTA b runs tile work[b].y of problem work[b].x, whose run
// description is copied from global memory into shared memory first. All
// problems of one launch share the tile shape, TB, sub0 and nsub.
template <typename T, int TB, int TI, int TJ, int NT, bool GEN>
__global__ void __launch_bounds__(NT) tm_tb_batch(const Dev<T>* devs, const int2* work, int sub0,
                                                  int nsub) {
  __shared__ __align__(16) unsigned char sdev[sizeof(Dev<T>)];
  const int2 w = work[blockIdx.x];
  const int* srcw = reinterpret_cast<const int*>(devs + w.x);
  for (int q = threadIdx.x; q < int(sizeof(Dev<T>) / sizeof(int)); q += NT)
    reinterpret_cast<int*>(sdev)[q] = srcw[q];
  __syncthreads();
  tb_body<T, TB, TI, TJ, NT, GEN>(*reinterpret_cast<const Dev<T>*>(sdev), w.y, sub0, nsub);
}

// ---------------------------------------------------------------------------
// Running DFT fold over `cnt` monitor-ring slots (fdtd2d.py:453-458): for
// each monitored cell, acc_k += sum_t ph[n0+t, k] x_t, partial sums in A.
// ---------------------------------------------------------------------------
template <typename T, typename A, int KM>
__global__ void __launch_bounds__(256) tm_dft_fold(Dev<T> d, int sub0, int cnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* sph = reinterpret_cast<A*>(smem_raw);  // [2 tables][cnt][K][re, im]
  using C = typename Cplx<A>::type;
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
  // Ring cells of all monitors form one index space (monitor m holds
  // [off_m, off_m + count_m)); each thread finds its monitor by binary search.
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
  const MonD mon = d.mons[lo];
  const long long loc = r - mon.off;
  const A* ph = sph + (mon.comp == 0 ? 0 : 2 * cnt * K);
  A are[KM], aim[KM];
#pragma unroll
  for (int k = 0; k < KM; ++k) are[k] = aim[k] = A(0);
  const T* base = d.mring + r;
  // Eight ring loads in flight per thread, then their FMAs.
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
        for (int k = 0; k < KM; ++k) {
          if (k < K) {
            are[k] += pt[2 * k] * x[u];
            aim[k] += pt[2 * k + 1] * x[u];
          }
        }
      }
    }
    slot += 8;
    if (slot >= d.R) slot -= d.R;
  }
  C* acc = static_cast<C*>(mon.out) + loc;
#pragma unroll
  for (int k = 0; k < KM; ++k) {
    if (k < K) {
      C v = acc[(long long)k * mon.count];
      v.x += are[k];
      v.y += aim[k];
      acc[(long long)k * mon.count] = v;
    }
  }
}

// Total field energy 1/2 (eps Ez^2 + mu0 H^2) dA (fdtd2d.py:160-169) of the
// state after step n, reduced in double into eacc[2n], eacc[2n+1].
template <typename T>
__global__ void tm_energy(Dev<T> d, double* eacc, int sub) {
  const int n = *d.step_base + sub;
  const T* f = d.state[(n + 1) & 1];  // one step per launch: state after step n
  double ue = 0.0, uh = 0.0;
  const long long total = (long long)d.nx * d.ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = int(g / d.ny), j = int(g - (long long)i * d.ny);
    const long long c = cell_at(d.ld, i, j);
    const double e = double(f[c]);
    ue += double(d.eps[g]) * e * e;
    const double hx = double(f[d.plane + c]), hy = double(f[2 * d.plane + c]);
    uh += hx * hx + hy * hy;  // zero outside their grids
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

// Copy a caller (nx, ny) array into a padded plane (ca, cb at set-up).
template <typename T>
__global__ void tm_pad_in(const T* src, T* dst, int nx, int ny, int ld) {
  const long long total = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = int(g / ny), j = int(g - (long long)i * ny);
    dst[cell_at(ld, i, j)] = src[g];
  }
}

// Copy the final state slot into the caller's unpadded ez/hx/hy.
template <typename T>
__global__ void tm_copy_out(const T* slot, long long plane, int nx, int ny, int ld, T* ez, T* hx,
                            T* hy) {
  const long long total = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int i = int(g / ny), j = int(g - (long long)i * ny);
    const long long c = cell_at(ld, i, j);
    ez[g] = slot[c];
    if (j < ny - 1) hx[(long long)i * (ny - 1) + j] = slot[plane + c];
    if (i < nx - 1) hy[g] = slot[2 * plane + c];
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
  Cfg cfg;
  // Row march (tm_march) instead of shared-memory tiles (tm_tb): then a
  // "tile" is one warp's strip segment, cfg.ti its owned rows and cfg.tj its
  // owned columns.
  bool march = false;
  int ld = 0, rows = 0, tiles_x = 0, tiles_y = 0, n_tiles = 0, R = 32, n_gen = 0, n_int = 0;
  long long plane = 0, mon_cells = 0, n_mw = 0, n_mpts = 0;
  size_t state[2], ca, cb, psi[2], zero_end, tile_list, off[5], pts[5], mons, mw_off, mw, mring,
      step, eacc, tasks, mpts, total;
};

// The row march is selected with GDN_TM_KERNEL=march (runs that record the
// energy every step or are forced onto a tile shape keep the tile kernels).
// Measured on B200 at the 1024^2 benchmark workload it reaches 37-41
// Gcell-steps/s against 103 for the shared-memory tile kernels: with ~1000
// warps on 148 SMs each warp's row step is a long dependent chain, so the
// tiles stay the default.
static bool use_march(const GdnTmParams* p, int force_cfg) {
  if (p->record_energy || force_cfg >= 0) return false;
  const char* env = getenv("GDN_TM_KERNEL");
  return env && env[0] == 'm';
}

// Owned rows per march segment: GDN_TM_SEG, else 16 (8..64).
static int march_seg() {
  const char* env = getenv("GDN_TM_SEG");
  const int v = env ? atoi(env) : 16;
  return std::min(std::max(v, 8), march::SIMAX);
}

template <typename T>
static Cfg march_cfg() {
  return Cfg{march::TB, march_seg(), march::owned_cols<T>(), march::WPB * 32};
}

// Tile shape: one step per launch when the energy is recorded, else the
// largest TB=4 shape that still yields two CTAs per SM's worth of tiles.
static Cfg pick_cfg(const GdnTmParams* p, size_t esize, int force = -1) {
  if (p->record_energy) return kCfgStep;
  const Cfg* c = esize == sizeof(float) ? kCfgF32 : kCfgF64;
  if (force >= 0 && force < NCFG) return c[force];
  const char* env = getenv("GDN_TM_TILE");
  if (env && env[0] >= '0' && env[0] < '0' + NCFG && env[1] == 0) return c[env[0] - '0'];
  // Measured on B200 (f32, forward + adjoint at 1024^2 with the general
  // tiles skipping psi outside the slabs): 32x64 tiles 109 Gcell-steps/s,
  // 16x32 106, 64x64 102. Below a tile per SM for the 64x64 shape the 16x32
  // tiles keep more SMs busy (512^2: 47 vs 34; 140^2: 5.1 vs 2.7).
  const long long big = div_up(p->nx, c[0].ti) * div_up(p->ny, c[0].tj);
  return big >= 148 ? c[1] : c[2];
}

// Monitor boxes {comp, lo0, lo1, h, w} in ring order: the listed boxes, or
// the three full components when none are listed.
static std::vector<std::array<int, 5>> monitor_boxes(const GdnTmParams* p,
                                                     const GdnTmPoints* pts) {
  std::vector<std::array<int, 5>> v;
  if (p->n_freq <= 0) return v;
  if (p->n_monitors == 0) {
    v.push_back({0, 0, 0, p->nx, p->ny});
    v.push_back({1, 0, 0, p->nx, p->ny - 1});
    v.push_back({2, 0, 0, p->nx - 1, p->ny});
    return v;
  }
  for (int k = 0; k < p->n_monitors; ++k) {
    const GdnDftMonitor& m = pts->monitors[k];
    v.push_back({m.comp, m.lo[0], m.lo[1], m.hi[0] - m.lo[0], m.hi[1] - m.lo[1]});
  }
  return v;
}

static long long monitor_cells(const GdnTmParams* p, const GdnTmPoints* pts) {
  long long c = 0;
  for (const auto& b : monitor_boxes(p, pts)) c += (long long)b[3] * b[4];
  return c;
}

// Number of (tile, monitor) parts: every tile a monitor box crosses.
static long long monitor_parts(const GdnTmParams* p, const GdnTmPoints* pts, const Cfg& c) {
  long long n = 0;
  for (const auto& b : monitor_boxes(p, pts))
    if (b[3] > 0 && b[4] > 0)
      n += (long long)((b[1] + b[3] - 1) / c.ti - b[1] / c.ti + 1) *
           ((b[2] + b[4] - 1) / c.tj - b[2] / c.tj + 1);
  return n;
}

// Interior tiles: every cell of the extended region is an interior Ez cell
// outside all CPML slabs (x slabs are i <= npml or i >= nx-1-npml, likewise
// y), so the interior kernel needs neither range checks nor psi. All other
// tiles are "general".
static bool tile_is_interior(const GdnTmParams* p, const Cfg& c, int ty, int tx) {
  const int m = p->npml;
  const int r0 = ty * c.ti - c.tb, r1 = (ty + 1) * c.ti + c.tb;
  const int c0 = tx * c.tj - HJ, c1 = (tx + 1) * c.tj + HJ;  // march: HJ == march::HJ
  return r0 >= m + 1 && r1 - 1 <= p->nx - 2 - m && c0 >= m + 1 && c1 - 1 <= p->ny - 2 - m;
}

// `ring_steps` > 0 forces the monitor-ring length (a multiple of TB).
static Layout make_layout(const GdnTmParams* p, const GdnTmPoints* pts, size_t esize,
                          int ring_steps = 0, int force_cfg = -1) {
  Layout L;
  L.march = use_march(p, force_cfg);
  L.cfg = L.march ? (esize == sizeof(float) ? march_cfg<float>() : march_cfg<double>())
                  : pick_cfg(p, esize, force_cfg);
  const Cfg& c = L.cfg;
  L.tiles_x = int(div_up(p->ny, c.tj));
  L.tiles_y = int(div_up(p->nx, c.ti));
  L.n_tiles = L.tiles_x * L.tiles_y;
  L.ld = PADJ + L.tiles_x * c.tj + PADJ;
  L.rows = L.tiles_y * c.ti + 2 * PADI;
  L.plane = (long long)L.rows * L.ld;
  // Without a monitor list (n_monitors == 0) a DFT records the full grid;
  // the points are only read for listed monitors, so pts may be NULL then.
  const bool mons_known = pts || p->n_monitors == 0;
  L.mon_cells = mons_known ? monitor_cells(p, pts) : 0;
  L.n_mw = mons_known ? monitor_parts(p, pts, c) : 0;
  if (ring_steps > 0) {
    L.R = ring_steps;
  } else {
    const size_t budget = size_t(2) << 30;  // monitor ring budget: 2 GiB
    long long r = L.mon_cells > 0 ? (long long)(budget / (size_t(L.mon_cells) * esize)) : 32;
    r = std::min<long long>(32, r);
    r = std::max<long long>(c.tb, r - r % c.tb);
    L.R = int(r);
  }
  for (int ty = 0; ty < L.tiles_y; ++ty)
    for (int tx = 0; tx < L.tiles_x; ++tx) {
      if (tile_is_interior(p, c, ty, tx))
        ++L.n_int;
      else
        ++L.n_gen;
    }
  Carve cv;
  // Everything up to zero_end is cleared at the start of a run.
  for (int s = 0; s < 2; ++s) L.state[s] = cv.take<char>(3 * size_t(L.plane) * esize);
  L.ca = cv.take<char>(size_t(L.plane) * esize);
  L.cb = cv.take<char>(size_t(L.plane) * esize);
  for (int s = 0; s < 2; ++s) L.psi[s] = cv.take<char>(4 * size_t(L.plane) * esize);
  L.step = cv.take<int>(1);
  L.zero_end = cv.take<char>(0);
  L.tile_list = cv.take<int>(L.n_tiles);  // general tiles first, then interior
  const int counts[5] = {p->n_sources, p->n_ports, p->n_mx, p->n_my, p->n_probes};
  if (L.march) {
    // A point lies in the extended range of at most two segments x two strips.
    long long np = 0;
    for (int k = 0; k < 5; ++k) np += counts[k];
    L.n_mpts = 4 * np;
    L.tasks = cv.take<MTask>(size_t(L.n_tiles));
    L.mpts = cv.take<MPt>(size_t(std::max<long long>(L.n_mpts, 1)));
  } else {
    for (int k = 0; k < 5; ++k) {
      L.off[k] = cv.take<int>(L.n_tiles + 1);
      L.pts[k] = cv.take<Pt>(4 * size_t(std::max(counts[k], 1)));
    }
  }
  L.mons = cv.take<MonD>(size_t(std::max(p->n_monitors, 3)));
  L.mw_off = cv.take<int>(L.n_tiles + 1);
  L.mw = cv.take<MonW>(size_t(std::max<long long>(L.n_mw, 1)));
  L.mring = cv.take<char>(std::max<size_t>(size_t(L.mon_cells) * L.R, 1) * esize);
  L.eacc = cv.take<double>(p->record_energy ? 2 * size_t(std::max(p->n_steps, 1)) : 1);
  L.total = cv.bytes();
  return L;
}

// Bin point records by every tile whose extended region holds the cell;
// `halo` = false keeps only the owner (probes). owner = 1 on the tile that
// owns the cell.
struct Bins {
  std::vector<int> off;
  std::vector<Pt> pts;
  int max_per_tile = 0;
};

static Bins bin_tiles(int n, const int32_t* pi, const int32_t* pj, const Layout& L, bool halo) {
  const Cfg& c = L.cfg;
  std::vector<std::pair<int, Pt>> rec;
  rec.reserve(4 * size_t(n));
  for (int m = 0; m < n; ++m) {
    const int i = pi[m], j = pj[m];
    const int oty = i / c.ti, otx = j / c.tj;
    for (int ty = std::max(0, oty - 1); ty <= std::min(L.tiles_y - 1, oty + 1); ++ty) {
      for (int tx = std::max(0, otx - 1); tx <= std::min(L.tiles_x - 1, otx + 1); ++tx) {
        const bool own = ty == oty && tx == otx;
        if (!own && !halo) continue;
        const int r0 = ty * c.ti - c.tb, r1 = (ty + 1) * c.ti + c.tb;
        const int c0 = tx * c.tj - HJ, c1 = (tx + 1) * c.tj + HJ;
        if (i < r0 || i >= r1 || j < c0 || j >= c1) continue;
        rec.push_back({ty * L.tiles_x + tx, Pt{m, i, j, own ? 1 : 0}});
      }
    }
  }
  std::stable_sort(rec.begin(), rec.end(),
                   [](const std::pair<int, Pt>& a, const std::pair<int, Pt>& b) {
                     return a.first < b.first;
                   });
  Bins b;
  b.off.assign(L.n_tiles + 1, 0);
  b.pts.resize(rec.size());
  for (size_t k = 0; k < rec.size(); ++k) {
    b.off[rec[k].first + 1]++;
    b.pts[k] = rec[k].second;
  }
  for (int t = 0; t < L.n_tiles; ++t) {
    b.max_per_tile = std::max(b.max_per_tile, b.off[t + 1]);
    b.off[t + 1] += b.off[t];
  }
  return b;
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
  if (p->n_monitors < 0) GDN_BAD_ARG("n_monitors must be >= 0");
  if (p->n_freq > 0 && p->n_monitors == 0 && (!b->dft_ez || !b->dft_hx || !b->dft_hy))
    GDN_BAD_ARG("dft output buffers are null");
  if (p->n_freq > 0 && p->n_monitors > 0) {
    if (!pts->monitors) GDN_BAD_ARG("monitor list is null");
    const int shp[3][2] = {{nx, ny}, {nx, ny - 1}, {nx - 1, ny}};
    for (int k = 0; k < p->n_monitors; ++k) {
      const GdnDftMonitor& m = pts->monitors[k];
      if (m.comp < 0 || m.comp > 2) GDN_BAD_ARG("monitor %d: component %d not in 0..2", k, m.comp);
      if (m.lo[0] < 0 || m.lo[1] < 0 || m.hi[0] > shp[m.comp][0] || m.hi[1] > shp[m.comp][1] ||
          m.hi[0] <= m.lo[0] || m.hi[1] <= m.lo[1])
        GDN_BAD_ARG("monitor %d: box [%d,%d)x[%d,%d) empty or outside component %d", k, m.lo[0],
                    m.hi[0], m.lo[1], m.hi[1], m.comp);
      if (!m.out) GDN_BAD_ARG("monitor %d: output is null", k);
    }
  }
  if (p->dt <= 0 || p->dx <= 0 || p->dy <= 0) GDN_BAD_ARG("dt, dx, dy must be positive");
  return GDN_OK;
}

// Everything one run needs on the device, filled by prepare().
template <typename T>
struct Run {
  Layout L;
  Dev<T> d{};
  std::vector<MonD> mons;
  long long max_cells = 0;
  double* eacc = nullptr;
  int* step_base = nullptr;
  const int* tiles = nullptr;  // L.n_gen general tile ids, then L.n_int interior
  // Row march: tasks in launch order (general first) and their tile ids.
  std::vector<MTask> mtasks;
  std::vector<int> mtask_tiles;
  const MTask* tasks = nullptr;
};

template <typename T>
static int prepare_tiles(const GdnTmParams* p, const GdnTmPoints* pts, char* ws, Run<T>& R,
                         cudaStream_t stream);
template <typename T>
static int prepare_march(const GdnTmParams* p, const GdnTmPoints* pts, char* ws, Run<T>& R,
                         cudaStream_t stream);
template <typename T>
static int prepare_common(const GdnTmParams* p, const GdnTmPoints* pts, const GdnTmBuffers* b,
                          char* ws, Run<T>& R, cudaStream_t stream);

template <typename T, int TB, int TI, int TJ, bool GEN>
static size_t tb_smem() {
  return size_t(GEN ? 9 : 5) * (TI + 2 * TB) * (TJ + 2 * HJ) * sizeof(T);
}

// Per-type tile configurations (compile-time copies of the tables).
template <typename T>
struct Kern;
template <>
struct Kern<float> {
  static constexpr const Cfg* c = kCfgF32;
};
template <>
struct Kern<double> {
  static constexpr const Cfg* c = kCfgF64;
};

template <typename T, int TB, int TI, int TJ, int NT, bool GEN>
static int set_attr() {
  const int sm = int(tb_smem<T, TB, TI, TJ, GEN>());
  GDN_TRY_CUDA(cudaFuncSetAttribute(tm_tb<T, TB, TI, TJ, NT, GEN>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  if constexpr (std::is_same<T, float>::value && TB > 1)
    GDN_TRY_CUDA(cudaFuncSetAttribute(tm_tb_batch<T, TB, TI, TJ, NT, GEN>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  return GDN_OK;
}

template <typename T, int I>
static int set_attr_cfg() {
  constexpr Cfg C = I < NCFG ? Kern<T>::c[I < NCFG ? I : 0] : kCfgStep;
  int st;
  if ((st = set_attr<T, C.tb, C.ti, C.tj, C.nt, true>())) return st;
  return set_attr<T, C.tb, C.ti, C.tj, C.nt, false>();
}

template <typename T>
static int set_kernel_attributes() {
  static bool done = false;  // per process; the attribute is per function
  if (done) return GDN_OK;
  int st;
  if ((st = set_attr_cfg<T, 0>()) || (st = set_attr_cfg<T, 1>()) || (st = set_attr_cfg<T, 2>()) ||
      (st = set_attr_cfg<T, 3>()) || (st = set_attr_cfg<T, 4>()) || (st = set_attr_cfg<T, NCFG>()))
    return st;
  GDN_TRY_CUDA(cudaFuncSetAttribute(march::tm_march<T, true, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(march::WPB * march::warp_smem<T, true, true>())));
  GDN_TRY_CUDA(cudaFuncSetAttribute(march::tm_march<T, false, false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(march::WPB * march::warp_smem<T, false, false>())));
  done = true;
  return GDN_OK;
}

// Index of a run's configuration in its type's table (NCFG: the one-step shape).
template <typename T>
static int cfg_index(const Cfg& c) {
  if (c.tb == 1) return NCFG;
  for (int i = 0; i < NCFG; ++i)
    if (Kern<T>::c[i].tb == c.tb && Kern<T>::c[i].ti == c.ti && Kern<T>::c[i].tj == c.tj)
      return i;
  return 0;
}

template <typename T, int TB, int TI, int TJ, int NT, bool GEN>
static void launch_cfg(const Run<T>& R, const int* tiles, int count, int sub0, int nsub,
                       cudaStream_t s) {
  tm_tb<T, TB, TI, TJ, NT, GEN>
      <<<count, NT, tb_smem<T, TB, TI, TJ, GEN>(), s>>>(R.d, tiles, sub0, nsub);
}

template <typename T, int I, bool GEN>
static void launch_idx(const Run<T>& R, const int* tiles, int count, int sub0, int nsub,
                       cudaStream_t s) {
  constexpr Cfg C = I < NCFG ? Kern<T>::c[I < NCFG ? I : 0] : kCfgStep;
  launch_cfg<T, C.tb, C.ti, C.tj, C.nt, GEN>(R, tiles, count, sub0, nsub, s);
}

template <typename T, bool GEN>
static void launch_which(int which, const Run<T>& R, const int* tiles, int count, int sub0,
                         int nsub, cudaStream_t s) {
  switch (which) {
    case 0: launch_idx<T, 0, GEN>(R, tiles, count, sub0, nsub, s); break;
    case 1: launch_idx<T, 1, GEN>(R, tiles, count, sub0, nsub, s); break;
    case 2: launch_idx<T, 2, GEN>(R, tiles, count, sub0, nsub, s); break;
    case 3: launch_idx<T, 3, GEN>(R, tiles, count, sub0, nsub, s); break;
    case 4: launch_idx<T, 4, GEN>(R, tiles, count, sub0, nsub, s); break;
    default: launch_idx<T, NCFG, GEN>(R, tiles, count, sub0, nsub, s); break;
  }
}

// Launch the general and the interior tiles for `nsub` steps starting at
// chunk offset `sub0`; with a side stream the two run concurrently.
template <typename T>
static uint64_t launch_tb(const Run<T>& R, int sub0, int nsub, cudaStream_t s, cudaStream_t side,
                          cudaEvent_t fork, cudaEvent_t join) {
  const int which = cfg_index<T>(R.L.cfg);
  const int ng = R.L.n_gen, ni = R.L.n_int;
  cudaStream_t si = s;
  if (side && ng > 0 && ni > 0) {
    cudaEventRecord(fork, s);
    cudaStreamWaitEvent(side, fork, 0);
    si = side;
  }
  uint64_t k = 0;
  if (R.L.march) {
    constexpr int W = march::WPB;
    if (ng > 0) {
      march::tm_march<T, true, true><<<unsigned(div_up(ng, W)), W * 32,
                                       W * march::warp_smem<T, true, true>(), s>>>(
          R.d, R.tasks, ng, sub0, nsub);
      ++k;
    }
    if (ni > 0) {
      march::tm_march<T, false, false><<<unsigned(div_up(ni, W)), W * 32,
                                         W * march::warp_smem<T, false, false>(), si>>>(
          R.d, R.tasks + ng, ni, sub0, nsub);
      ++k;
    }
  } else {
    if (ng > 0) {
      launch_which<T, true>(which, R, R.tiles, ng, sub0, nsub, s);
      ++k;
    }
    if (ni > 0) {
      launch_which<T, false>(which, R, R.tiles + ng, ni, sub0, nsub, si);
      ++k;
    }
  }
  if (si != s) {
    cudaEventRecord(join, side);
    cudaStreamWaitEvent(s, join, 0);
  }
  return k;
}

template <typename T, typename A>
static void launch_fold(const Run<T>& R, int cnt, int K, cudaStream_t s) {
  const unsigned dg = unsigned(div_up(R.L.mon_cells, 256));
  const size_t sm = size_t(4) * cnt * K * sizeof(A);
  if (K <= 4)
    tm_dft_fold<T, A, 4><<<dg, 256, sm, s>>>(R.d, 0, cnt);
  else if (K <= 8)
    tm_dft_fold<T, A, 8><<<dg, 256, sm, s>>>(R.d, 0, cnt);
  else
    tm_dft_fold<T, A, KMAX><<<dg, 256, sm, s>>>(R.d, 0, cnt);
}

// Enqueue one chunk of `cnt` steps (cnt <= R.L.R): step launches (+ energy),
// the DFT fold and the counter advance. Returns the number of kernels.
template <typename T>
static uint64_t enqueue_chunk(const Run<T>& R, const GdnTmParams* p, int cnt, cudaStream_t s,
                              cudaStream_t side = nullptr, cudaEvent_t fork = nullptr,
                              cudaEvent_t join = nullptr) {
  uint64_t k = 0;
  const int tb = R.L.cfg.tb;
  const int eblocks = int(std::min<long long>(div_up((long long)p->nx * p->ny, 256), 148 * 8));
  for (int sub = 0; sub < cnt; sub += tb) {
    k += launch_tb(R, sub, std::min(tb, cnt - sub), s, side, fork, join);
    if (p->record_energy) {  // tb == 1 here
      tm_energy<T><<<eblocks, 256, 0, s>>>(R.d, R.eacc, sub);
      ++k;
    }
  }
  if (!R.mons.empty()) {
    if (p->dft_f64)
      launch_fold<T, double>(R, cnt, p->n_freq, s);
    else
      launch_fold<T, float>(R, cnt, p->n_freq, s);
    ++k;
  }
  tm_advance<<<1, 1, 0, s>>>(R.step_base, cnt);
  return k + 1;
}

// Fill the device description, upload point bins and monitors, clear the
// state that starts at zero and pad ca/cb in. `ws` holds L.total bytes.
template <typename T>
static int prepare(const GdnTmParams* p, const GdnTmPoints* pts, const GdnTmBuffers* b, char* ws,
                   Run<T>& R, cudaStream_t stream) {
  const Layout& L = R.L;
  const int nx = p->nx, ny = p->ny, N = p->n_steps;
  Dev<T>& d = R.d;
  d.nx = nx;
  d.ny = ny;
  d.ld = L.ld;
  d.npml = p->npml;
  d.n_steps = N;
  d.n_freq = p->n_freq;
  d.R = L.R;
  d.tiles_x = L.tiles_x;
  d.plane = L.plane;
  d.state[0] = reinterpret_cast<T*>(ws + L.state[0]);
  d.state[1] = reinterpret_cast<T*>(ws + L.state[1]);
  d.mring = reinterpret_cast<T*>(ws + L.mring);
  d.mon_cells = L.mon_cells;
  d.ca = reinterpret_cast<const T*>(ws + L.ca);
  d.cb = reinterpret_cast<const T*>(ws + L.cb);
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
  for (int s = 0; s < 2; ++s) d.psi[s] = reinterpret_cast<T*>(ws + L.psi[s]);
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
  R.step_base = reinterpret_cast<int*>(ws + L.step);
  d.step_base = R.step_base;
  R.eacc = reinterpret_cast<double*>(ws + L.eacc);

  d.mpts = reinterpret_cast<const MPt*>(ws + L.mpts);
  int st = L.march ? prepare_march(p, pts, ws, R, stream) : prepare_tiles(p, pts, ws, R, stream);
  if (st) return st;
  return prepare_common(p, pts, b, ws, R, stream);
}

// Tile kernels: per-tile point bins and the general/interior tile lists.
template <typename T>
static int prepare_tiles(const GdnTmParams* p, const GdnTmPoints* pts, char* ws, Run<T>& R,
                         cudaStream_t stream) {
  const Layout& L = R.L;
  Dev<T>& d = R.d;
  // Point bins (with halo copies except for probes). Pageable copies are
  // staged before cudaMemcpyAsync returns, so the vectors may go away.
  const int counts[5] = {p->n_sources, p->n_ports, p->n_mx, p->n_my, p->n_probes};
  const int32_t* is[5] = {pts->src_i, pts->port_i, pts->mx_i, pts->my_i, pts->probe_i};
  const int32_t* js[5] = {pts->src_j, pts->port_j, pts->mx_j, pts->my_j, pts->probe_j};
  const int* offs[5];
  const Pt* pls[5];
  for (int k = 0; k < 5; ++k) {
    Bins bn = bin_tiles(counts[k], is[k], js[k], L, k != 4);
    if (k == 1 && bn.max_per_tile > MAXP)
      GDN_BAD_ARG("%d port records fall in one tile (at most %d)", bn.max_per_tile, MAXP);
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.off[k], bn.off.data(), bn.off.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    if (!bn.pts.empty())
      GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.pts[k], bn.pts.data(), bn.pts.size() * sizeof(Pt),
                                   cudaMemcpyHostToDevice, stream));
    offs[k] = reinterpret_cast<const int*>(ws + L.off[k]);
    pls[k] = reinterpret_cast<const Pt*>(ws + L.pts[k]);
  }
  d.src_off = offs[0]; d.src_pts = pls[0];
  d.port_off = offs[1]; d.port_pts = pls[1];
  d.mx_off = offs[2]; d.mx_pts = pls[2];
  d.my_off = offs[3]; d.my_pts = pls[3];
  d.probe_off = offs[4]; d.probe_pts = pls[4];

  // Tile lists: general tiles first, then interior tiles.
  {
    std::vector<int> gen, inr;
    for (int ty = 0; ty < L.tiles_y; ++ty)
      for (int tx = 0; tx < L.tiles_x; ++tx)
        (tile_is_interior(p, L.cfg, ty, tx) ? inr : gen).push_back(ty * L.tiles_x + tx);
    gen.insert(gen.end(), inr.begin(), inr.end());
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.tile_list, gen.data(), gen.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    R.tiles = reinterpret_cast<const int*>(ws + L.tile_list);
  }
  return GDN_OK;
}

// Row march: one task per (segment, strip), general tasks first; every
// point's copies in each task whose extended range holds it, sorted by task,
// row and type (the order a step applies them).
template <typename T>
static int prepare_march(const GdnTmParams* p, const GdnTmPoints* pts, char* ws, Run<T>& R,
                         cudaStream_t stream) {
  const Layout& L = R.L;
  const Cfg& c = L.cfg;
  const int SI = c.ti, OW = c.tj, TBm = march::TB, HJm = march::HJ;
  const int SW = OW + 2 * HJm;  // strip width (32 * V)
  std::vector<int> order;
  order.reserve(L.n_tiles);
  for (int pass = 0; pass < 2; ++pass)
    for (int ty = 0; ty < L.tiles_y; ++ty)
      for (int tx = 0; tx < L.tiles_x; ++tx)
        if (tile_is_interior(p, c, ty, tx) == (pass == 1)) order.push_back(ty * L.tiles_x + tx);
  std::vector<int> pos(L.n_tiles);
  for (int k = 0; k < L.n_tiles; ++k) pos[order[k]] = k;
  struct Rec {
    int task;
    MPt e;
  };
  std::vector<Rec> rec;
  rec.reserve(size_t(L.n_mpts));
  const int counts[5] = {p->n_mx, p->n_my, p->n_ports, p->n_sources, p->n_probes};
  const int32_t* is[5] = {pts->mx_i, pts->my_i, pts->port_i, pts->src_i, pts->probe_i};
  const int32_t* js[5] = {pts->mx_j, pts->my_j, pts->port_j, pts->src_j, pts->probe_j};
  const int types[5] = {march::P_MX, march::P_MY, march::P_PORT, march::P_SRC, march::P_PROBE};
  for (int k = 0; k < 5; ++k) {
    for (int m = 0; m < counts[k]; ++m) {
      const int i = is[k][m], j = js[k][m];
      const int oty = i / SI, otx = j / OW;
      for (int ty = std::max(0, oty - 1); ty <= std::min(L.tiles_y - 1, oty + 1); ++ty)
        for (int tx = std::max(0, otx - 1); tx <= std::min(L.tiles_x - 1, otx + 1); ++tx) {
          const bool own = ty == oty && tx == otx;
          if (!own && types[k] == march::P_PROBE) continue;
          const int r0 = ty * SI - TBm, r1 = (ty + 1) * SI + TBm;
          const int c0 = tx * OW - HJm, c1 = c0 + SW;
          if (i < r0 || i >= r1 || j < c0 || j >= c1) continue;
          rec.push_back({pos[ty * L.tiles_x + tx], MPt{i, j, m, types[k] | (own ? 8 : 0)}});
        }
    }
  }
  if ((long long)rec.size() > std::max<long long>(L.n_mpts, 1))
    GDN_BAD_ARG("internal: %zu point entries, layout sized for %lld", rec.size(), L.n_mpts);
  std::stable_sort(rec.begin(), rec.end(), [](const Rec& a, const Rec& b) {
    if (a.task != b.task) return a.task < b.task;
    if (a.e.i != b.e.i) return a.e.i < b.e.i;
    return (a.e.tag & 7) < (b.e.tag & 7);
  });
  std::vector<MPt> ent(rec.size());
  std::vector<int> off(L.n_tiles + 1, 0);
  for (size_t k = 0; k < rec.size(); ++k) {
    ent[k] = rec[k].e;
    off[rec[k].task + 1]++;
  }
  for (int t = 0; t < L.n_tiles; ++t) off[t + 1] += off[t];
  R.mtask_tiles = order;
  R.mtasks.assign(L.n_tiles, MTask{});
  for (int k = 0; k < L.n_tiles; ++k) {
    const int t = order[k], ty = t / L.tiles_x, tx = t - ty * L.tiles_x;
    MTask& tk = R.mtasks[k];
    tk.i0 = ty * SI;
    tk.j0 = tx * OW;
    tk.rows = std::min(SI, p->nx - tk.i0);
    tk.cls = k < L.n_gen ? 1 : 0;
    tk.pb = off[k];
    tk.pe = off[k + 1];
    tk.mb = tk.me = 0;  // filled by prepare_common from the monitor parts
  }
  if (!ent.empty())
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.mpts, ent.data(), ent.size() * sizeof(MPt),
                                 cudaMemcpyHostToDevice, stream));
  R.tasks = reinterpret_cast<const MTask*>(ws + L.tasks);
  return GDN_OK;
}

// Monitors, monitor parts, DFT output clears, state clears and ca/cb padding.
template <typename T>
static int prepare_common(const GdnTmParams* p, const GdnTmPoints* pts, const GdnTmBuffers* b,
                          char* ws, Run<T>& R, cudaStream_t stream) {
  const Layout& L = R.L;
  Dev<T>& d = R.d;
  const int nx = p->nx, ny = p->ny, N = p->n_steps;

  // Monitors (full grid when none are listed).
  const bool f64acc = p->dft_f64 != 0;
  const size_t csz = f64acc ? sizeof(double2) : sizeof(float2);
  R.mons.clear();
  {
    void* const full_out[3] = {b->dft_ez, b->dft_hx, b->dft_hy};
    long long off = 0;
    int k = 0;
    for (const auto& bx : monitor_boxes(p, pts)) {
      void* out = p->n_monitors == 0 ? full_out[k] : pts->monitors[k].out;
      const long long cnt = (long long)bx[3] * bx[4];
      R.mons.push_back(MonD{bx[0], bx[1], bx[2], bx[3], bx[4], 0, cnt, off, out});
      off += cnt;
      ++k;
    }
  }
  d.n_mons = int(R.mons.size());
  d.mons = reinterpret_cast<const MonD*>(ws + L.mons);
  // Monitor parts per tile (CSR), in tile order.
  {
    const Cfg& c = L.cfg;
    std::vector<std::vector<MonW>> per(L.n_tiles);
    for (const MonD& m : R.mons) {
      if (m.h <= 0 || m.w <= 0) continue;
      for (int ty = m.lo0 / c.ti; ty <= (m.lo0 + m.h - 1) / c.ti; ++ty)
        for (int tx = m.lo1 / c.tj; tx <= (m.lo1 + m.w - 1) / c.tj; ++tx) {
          MonW e;
          e.a0 = std::max(m.lo0, ty * c.ti);
          e.a1 = std::min(m.lo0 + m.h, (ty + 1) * c.ti);
          e.b0 = std::max(m.lo1, tx * c.tj);
          e.b1 = std::min(m.lo1 + m.w, (tx + 1) * c.tj);
          e.comp = m.comp;
          e.w = m.w;
          e.base = m.off - (long long)m.lo0 * m.w - m.lo1;
          per[ty * L.tiles_x + tx].push_back(e);
        }
    }
    std::vector<int> moff(L.n_tiles + 1, 0);
    std::vector<MonW> mw;
    mw.reserve(size_t(L.n_mw));
    for (int t = 0; t < L.n_tiles; ++t) {
      mw.insert(mw.end(), per[t].begin(), per[t].end());
      moff[t + 1] = int(mw.size());
    }
    if ((long long)mw.size() != L.n_mw)
      GDN_BAD_ARG("internal: %zu monitor parts, layout sized for %lld", mw.size(), L.n_mw);
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.mw_off, moff.data(), moff.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    if (!mw.empty())
      GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.mw, mw.data(), mw.size() * sizeof(MonW),
                                   cudaMemcpyHostToDevice, stream));
    d.mw_off = reinterpret_cast<const int*>(ws + L.mw_off);
    d.mw = reinterpret_cast<const MonW*>(ws + L.mw);
    if (L.march) {
      for (size_t k = 0; k < R.mtasks.size(); ++k) {
        const int t = R.mtask_tiles[k];
        R.mtasks[k].mb = moff[t];
        R.mtasks[k].me = moff[t + 1];
      }
      GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.tasks, R.mtasks.data(), R.mtasks.size() * sizeof(MTask),
                                   cudaMemcpyHostToDevice, stream));
    }
  }
  R.max_cells = 0;
  for (const MonD& m : R.mons) {
    R.max_cells = std::max(R.max_cells, m.count);
    GDN_TRY_CUDA(cudaMemsetAsync(m.out, 0, size_t(m.count) * p->n_freq * csz, stream));
  }
  if (!R.mons.empty())
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + L.mons, R.mons.data(), R.mons.size() * sizeof(MonD),
                                 cudaMemcpyHostToDevice, stream));

  // Clear the state that starts at zero: both field slots (ghost cells
  // included), padded ca/cb, both psi parities, the step counter.
  GDN_TRY_CUDA(cudaMemsetAsync(ws + L.state[0], 0, L.zero_end - L.state[0], stream));
  if (p->record_energy)
    GDN_TRY_CUDA(cudaMemsetAsync(R.eacc, 0, 2 * size_t(std::max(N, 1)) * sizeof(double), stream));
  const int eblocks = int(std::min<long long>(div_up((long long)nx * ny, 256), 148 * 8));
  tm_pad_in<T><<<eblocks, 256, 0, stream>>>(static_cast<const T*>(b->ca),
                                             reinterpret_cast<T*>(ws + L.ca), nx, ny, L.ld);
  tm_pad_in<T><<<eblocks, 256, 0, stream>>>(static_cast<const T*>(b->cb),
                                             reinterpret_cast<T*>(ws + L.cb), nx, ny, L.ld);
  count_launches(2);
  return GDN_OK;
}

// Copy the final fields out, scale the DFT by dt (fdtd2d.py:482-487), finish
// the energy record.
template <typename T>
static int finalize(const GdnTmParams* p, const GdnTmBuffers* b, const Run<T>& R,
                    cudaStream_t stream) {
  const int nx = p->nx, ny = p->ny, N = p->n_steps;
  const long long launches = div_up(N, R.L.cfg.tb);
  const T* last = R.d.state[launches & 1];
  const int eblocks = int(std::min<long long>(div_up((long long)nx * ny, 256), 148 * 8));
  tm_copy_out<T><<<eblocks, 256, 0, stream>>>(last, R.L.plane, nx, ny, R.L.ld,
                                              static_cast<T*>(b->ez), static_cast<T*>(b->hx),
                                              static_cast<T*>(b->hy));
  for (const MonD& m : R.mons) {
    const long long cnt = m.count * p->n_freq;
    const int blocks = int(std::min<long long>(div_up(cnt, 256), 148 * 8));
    if (p->dft_f64)
      tm_dft_scale<double2><<<blocks, 256, 0, stream>>>(static_cast<double2*>(m.out), cnt, p->dt);
    else
      tm_dft_scale<float2><<<blocks, 256, 0, stream>>>(static_cast<float2*>(m.out), cnt, p->dt);
  }
  if (p->record_energy && N > 0)
    tm_energy_finish<T><<<unsigned(div_up(N, 256)), 256, 0, stream>>>(
        R.eacc, static_cast<T*>(b->out_energy), N, p->dx * p->dy, p->mu0);
  count_launches(1 + R.mons.size() + (p->record_energy && N > 0 ? 1 : 0));
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}

template <typename T>
static int run(const GdnTmParams* p, const GdnTmPoints* pts, const GdnTmBuffers* b,
               cudaStream_t stream) {
  int st = validate(p, pts, b);
  if (st) return st;
  if ((st = set_kernel_attributes<T>())) return st;
  Run<T> R;
  R.L = make_layout(p, pts, sizeof(T));
  char* ws = static_cast<char*>(b->workspace);
  bool own = false;
  if (!ws) {
    GDN_TRY_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ws), R.L.total, stream));
    own = true;
  } else if (b->workspace_bytes < R.L.total) {
    GDN_BAD_ARG("workspace too small: %zu < %zu bytes", b->workspace_bytes, R.L.total);
  }
  struct Guard {
    char* p;
    bool own;
    cudaStream_t s;
    ~Guard() {
      if (own && p) cudaFreeAsync(p, s);
    }
  } guard{ws, own, stream};
  if ((st = prepare(p, pts, b, ws, R, stream))) return st;

  // Capture one chunk of `cnt` steps as a graph; the general and interior
  // tile launches of each block become parallel branches.
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  GDN_TRY_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  GDN_TRY_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } ev_guard{ev_fork, ev_join};
  uint64_t per_chunk = 0;
  auto capture = [&](int cnt, cudaGraphExec_t* exec) -> int {
    cudaStream_t cs = capture_stream();
    if (!cs) GDN_BAD_ARG("no capture stream for this device");
    cudaStream_t side = capture_side_stream();
    GDN_TRY_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    per_chunk = enqueue_chunk(R, p, cnt, cs, side, ev_fork, ev_join);
    cudaGraph_t g = nullptr;
    const cudaError_t e1 = cudaStreamEndCapture(cs, &g);
    if (e1 != cudaSuccess) {
      set_error("graph capture failed: %s", cudaGetErrorString(e1));
      return GDN_ERR_CUDA;
    }
    const cudaError_t e2 = cudaGraphInstantiate(exec, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
      set_error("graph instantiate failed: %s", cudaGetErrorString(e2));
      return GDN_ERR_CUDA;
    }
    return GDN_OK;
  };
  const int N = p->n_steps, Tc = R.L.R;
  const int full = N / Tc, rem = N % Tc;
  cudaGraphExec_t g_full = nullptr, g_rem = nullptr;
  uint64_t k_full = 0, k_rem = 0;
  if (full > 0) {
    if ((st = capture(Tc, &g_full))) return st;
    k_full = per_chunk;
  }
  if (rem > 0) {
    if ((st = capture(rem, &g_rem))) {
      if (g_full) cudaGraphExecDestroy(g_full);
      return st;
    }
    k_rem = per_chunk;
  }
  cudaError_t le = cudaSuccess;
  const int tbd = R.L.cfg.tb;
  LoopTimer timer(stream, double(p->nx) * p->ny * N,
                  int64_t(full) * div_up(Tc, tbd) + div_up(rem, tbd));
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
  return finalize(p, b, R, stream);
}


// ---------------------------------------------------------------------------
// Batched runs: many independent problems advanced by shared launches.
// ---------------------------------------------------------------------------

template <int I>
static void launch_batch_idx(bool gen, const Dev<float>* devs, const int2* work, int count,
                             int sub0, int nsub, cudaStream_t s) {
  constexpr Cfg C = kCfgF32[I];
  if (gen)
    tm_tb_batch<float, C.tb, C.ti, C.tj, C.nt, true>
        <<<count, C.nt, tb_smem<float, C.tb, C.ti, C.tj, true>(), s>>>(devs, work, sub0, nsub);
  else
    tm_tb_batch<float, C.tb, C.ti, C.tj, C.nt, false>
        <<<count, C.nt, tb_smem<float, C.tb, C.ti, C.tj, false>(), s>>>(devs, work, sub0, nsub);
}

static void launch_batch(int which, bool gen, const Dev<float>* devs, const int2* work, int count,
                         int sub0, int nsub, cudaStream_t s) {
  switch (which) {
    case 0: launch_batch_idx<0>(gen, devs, work, count, sub0, nsub, s); break;
    case 1: launch_batch_idx<1>(gen, devs, work, count, sub0, nsub, s); break;
    case 2: launch_batch_idx<2>(gen, devs, work, count, sub0, nsub, s); break;
    case 3: launch_batch_idx<3>(gen, devs, work, count, sub0, nsub, s); break;
    default: launch_batch_idx<4>(gen, devs, work, count, sub0, nsub, s); break;
  }
}

// All problems share one tile configuration (`cfg`, or the heuristic for the
// largest problem) and one monitor-ring length, so chunk boundaries line up;
// each keeps its own grid, CPML, sources, ports, monitors and step count.
// Per block launch the work list holds (problem, tile) pairs of the problems
// still running, ordered by decreasing step count so the active ones are a
// prefix; a problem whose last block is partial gets its own launch.
static int run_batch_f32(const GdnTmProblem* probs, int n, int cfg, cudaStream_t stream) {
  using T = float;
  if (n < 0 || (n > 0 && !probs)) GDN_BAD_ARG("invalid problem list");
  if (cfg < -1 || cfg >= NCFG) GDN_BAD_ARG("cfg %d outside [-1, %d)", cfg, NCFG);
  if (n == 0) return GDN_OK;
  int st;
  if ((st = set_kernel_attributes<T>())) return st;
  // Configuration and common ring length.
  int big = 0;
  for (int q = 0; q < n; ++q) {
    const GdnTmProblem& pr = probs[q];
    if ((st = validate(pr.params, pr.points, pr.buffers))) {
      const std::string msg = last_error();
      GDN_BAD_ARG("problem %d: %s", q, msg.c_str());
    }
    if (pr.params->record_energy) GDN_BAD_ARG("problem %d: batched runs do not record the energy", q);
    const GdnTmParams* a = pr.params;
    const GdnTmParams* b0 = probs[big].params;
    if ((long long)a->nx * a->ny > (long long)b0->nx * b0->ny) big = q;
  }
  const int which = cfg >= 0 ? cfg : cfg_index<T>(pick_cfg(probs[big].params, sizeof(T)));
  std::vector<Run<T>> R(n);
  int ring = 1 << 30;
  for (int q = 0; q < n; ++q) {
    R[q].L = make_layout(probs[q].params, probs[q].points, sizeof(T), 0, which);
    ring = std::min(ring, R[q].L.R);
  }
  const int tb = kCfgF32[which].tb;
  // Workspaces (the caller's, or one stream-ordered block for the rest) and
  // a device block for the run descriptors and work lists.
  std::vector<size_t> woff(n, 0);
  size_t own_bytes = 0;
  for (int q = 0; q < n; ++q) {
    if (R[q].L.R != ring)
      R[q].L = make_layout(probs[q].params, probs[q].points, sizeof(T), ring, which);
    const GdnTmBuffers* b = probs[q].buffers;
    if (b->workspace) {
      if (b->workspace_bytes < R[q].L.total)
        GDN_BAD_ARG("problem %d: workspace too small: %zu < %zu bytes", q, b->workspace_bytes,
                    R[q].L.total);
    } else {
      woff[q] = own_bytes;
      own_bytes += (R[q].L.total + 255) & ~size_t(255);
    }
  }
  // Order by decreasing step count; work lists per tile class.
  std::vector<int> order(n);
  for (int q = 0; q < n; ++q) order[q] = q;
  std::stable_sort(order.begin(), order.end(), [&](int u, int v) {
    return probs[u].params->n_steps > probs[v].params->n_steps;
  });
  std::vector<int2> wgen, wint;
  std::vector<int> gpos(n + 1, 0), ipos(n + 1, 0);  // prefix positions in `order` order
  for (int r = 0; r < n; ++r) {
    const int q = order[r];
    const GdnTmParams* p = probs[q].params;
    const Layout& L = R[q].L;
    gpos[r] = int(wgen.size());
    ipos[r] = int(wint.size());
    for (int ty = 0; ty < L.tiles_y; ++ty)
      for (int tx = 0; tx < L.tiles_x; ++tx)
        (tile_is_interior(p, L.cfg, ty, tx) ? wint : wgen).push_back(make_int2(q, ty * L.tiles_x + tx));
  }
  gpos[n] = int(wgen.size());
  ipos[n] = int(wint.size());
  const size_t dev_bytes = size_t(n) * sizeof(Dev<T>);
  const size_t aux = ((dev_bytes + 255) & ~size_t(255)) + (wgen.size() + wint.size() + 2) * sizeof(int2);
  char* block = nullptr;
  GDN_TRY_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&block), own_bytes + aux + 256, stream));
  struct Guard {
    char* p;
    cudaStream_t s;
    ~Guard() {
      if (p) cudaFreeAsync(p, s);
    }
  } guard{block, stream};
  char* aux_base = block + ((own_bytes + 255) & ~size_t(255));
  Dev<T>* d_devs = reinterpret_cast<Dev<T>*>(aux_base);
  int2* d_gen = reinterpret_cast<int2*>(aux_base + ((dev_bytes + 255) & ~size_t(255)));
  int2* d_int = d_gen + wgen.size() + 1;
  // Prepare every problem in its workspace.
  std::vector<Dev<T>> hdev(n);
  for (int q = 0; q < n; ++q) {
    const GdnTmBuffers* b = probs[q].buffers;
    char* ws = b->workspace ? static_cast<char*>(b->workspace) : block + woff[q];
    if ((st = prepare(probs[q].params, probs[q].points, b, ws, R[q], stream))) {
      const std::string msg = last_error();
      GDN_BAD_ARG("problem %d: %s", q, msg.c_str());
    }
    hdev[q] = R[q].d;
  }
  GDN_TRY_CUDA(cudaMemcpyAsync(d_devs, hdev.data(), dev_bytes, cudaMemcpyHostToDevice, stream));
  if (!wgen.empty())
    GDN_TRY_CUDA(cudaMemcpyAsync(d_gen, wgen.data(), wgen.size() * sizeof(int2),
                                 cudaMemcpyHostToDevice, stream));
  if (!wint.empty())
    GDN_TRY_CUDA(cudaMemcpyAsync(d_int, wint.data(), wint.size() * sizeof(int2),
                                 cudaMemcpyHostToDevice, stream));
  // The host arrays above are pageable: cudaMemcpyAsync has staged them when
  // it returns, so the vectors may be reused below.
  int nmax = 0;
  double cell_steps = 0;
  int64_t blocks = 0;
  for (int q = 0; q < n; ++q) {
    const GdnTmParams* p = probs[q].params;
    nmax = std::max(nmax, p->n_steps);
    cell_steps += double(p->nx) * p->ny * p->n_steps;
    blocks += div_up(p->n_steps, tb);
  }
  uint64_t launches = 0;
  LoopTimer timer(stream, cell_steps, blocks);
  auto launch_range = [&](int r0, int r1, int sub, int nsub) {
    const int g0 = gpos[r0], g1 = gpos[r1], i0 = ipos[r0], i1 = ipos[r1];
    if (g1 > g0) {
      launch_batch(which, true, d_devs, d_gen + g0, g1 - g0, sub, nsub, stream);
      ++launches;
    }
    if (i1 > i0) {
      launch_batch(which, false, d_devs, d_int + i0, i1 - i0, sub, nsub, stream);
      ++launches;
    }
  };
  for (int base = 0; base < nmax; base += ring) {
    for (int sub = 0; sub < ring && base + sub < nmax; sub += tb) {
      // Problems with a full block here form a prefix of `order`.
      int full = 0;
      while (full < n && probs[order[full]].params->n_steps - base - sub >= tb) ++full;
      launch_range(0, full, sub, tb);
      // Then the problems whose last block this is, one launch each.
      for (int r = full; r < n; ++r) {
        const int left = probs[order[r]].params->n_steps - base - sub;
        if (left <= 0) break;
        launch_range(r, r + 1, sub, left);
      }
    }
    for (int r = 0; r < n; ++r) {
      const int q = order[r];
      const GdnTmParams* p = probs[q].params;
      const int cnt = std::min(ring, p->n_steps - base);
      if (cnt <= 0) break;
      if (!R[q].mons.empty()) {
        if (p->dft_f64)
          launch_fold<T, double>(R[q], cnt, p->n_freq, stream);
        else
          launch_fold<T, float>(R[q], cnt, p->n_freq, stream);
        ++launches;
      }
      tm_advance<<<1, 1, 0, stream>>>(R[q].step_base, cnt);
      ++launches;
    }
  }
  const cudaError_t le = cudaGetLastError();
  timer.stop(le == cudaSuccess);
  if (le != cudaSuccess) {
    set_error("batched launch failed: %s", cudaGetErrorString(le));
    return GDN_ERR_CUDA;
  }
  count_launches(launches);
  for (int q = 0; q < n; ++q)
    if ((st = finalize(probs[q].params, probs[q].buffers, R[q], stream))) return st;
  return GDN_OK;
}

}  // namespace tm2d
}  // namespace gdn

extern "C" int gdn_tm_workspace_size(const GdnTmParams* p, const GdnTmPoints* pts, int f64,
                                     size_t* bytes) {
  if (!p || !bytes) {
    gdn::set_error("null argument");
    return GDN_ERR_BAD_ARG;
  }
  if (p->nx < 3 || p->ny < 3 || p->npml < 0) {
    gdn::set_error("invalid grid");
    return GDN_ERR_BAD_ARG;
  }
  if (p->n_freq > 0 && p->n_monitors > 0 && (!pts || !pts->monitors)) {
    gdn::set_error("monitor list is null");
    return GDN_ERR_BAD_ARG;
  }
  *bytes = gdn::tm2d::make_layout(p, pts, f64 ? sizeof(double) : sizeof(float)).total;
  return GDN_OK;
}

extern "C" int gdn_tm_run_f32(const GdnTmParams* p, const GdnTmPoints* pts,
                              const GdnTmBuffers* b, void* stream) {
  return gdn::tm2d::run<float>(p, pts, b, static_cast<cudaStream_t>(stream));
}

extern "C" int gdn_tm_run_batch_f32(const GdnTmProblem* problems, int32_t n, int32_t cfg,
                                    void* stream) {
  return gdn::tm2d::run_batch_f32(problems, n, cfg, static_cast<cudaStream_t>(stream));
}

extern "C" int gdn_tm_run_f64(const GdnTmParams* p, const GdnTmPoints* pts,
                              const GdnTmBuffers* b, void* stream) {
  return gdn::tm2d::run<double>(p, pts, b, static_cast<cudaStream_t>(stream));
}

// ===========================================================================
// Allocation-free 2D TM entry point (no counterpart in the reference).
//
// For callers that cannot allocate device memory while they run the solver:
// code that owns the GPU's memory through its own pool (the allocation would
// fail or fragment that pool), real-time loops that forbid allocator calls,
// and hosts that load this library without a CUDA allocator they may use.
// The scratch (field state, psi slabs, point bins, monitor table and ring,
// step counter) lives in one file-scope __device__ array of fixed size
// instead of a workspace. Every GPU that loads this library holds the array
// until the process exits.
// ===========================================================================
namespace gdn {
namespace tm2d {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;  // 32 MiB per device
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch on the current device. In host code the
// array's name is only a host-side stand-in, so every call looks the address
// up with cudaGetSymbolAddress, with the caller's device current. The lookup
// is cheap and allocates nothing once the module is loaded; doing it on every
// call (instead of caching it) keeps the address right after a device reset,
// which reloads the module elsewhere. With CUDA's lazy module loading, the
// first lookup on a device loads this library's module, which reserves the
// array itself (and the module's code) on that device.
static int static_scratch(char** out) {
  void* p = nullptr;
  GDN_TRY_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
  *out = static_cast<char*>(p);
  return GDN_OK;
}

// The gdn_tm_run_f32 time loop with the static scratch, launched eagerly
// (no CUDA graph is instantiated, since instantiation may allocate).
static int run_noalloc_f32(const GdnTmParams* p, const GdnTmPoints* pts, const GdnTmBuffers* b,
                           cudaStream_t stream) {
  using T = float;
  int st = validate(p, pts, b);
  if (st) return st;
  if ((st = set_kernel_attributes<T>())) return st;
  // Largest monitor-ring length (a multiple of TB) whose layout fits.
  Run<T> R;
  R.L = make_layout(p, pts, sizeof(T));
  const int tb = R.L.cfg.tb;
  for (int r = R.L.R; r > tb && R.L.total > kStaticScratchBytes; r -= tb)
    R.L = make_layout(p, pts, sizeof(T), r - tb);
  if (R.L.total > kStaticScratchBytes)
    GDN_BAD_ARG("this run needs %zu bytes of scratch; the static scratch of "
                "gdn_tm_run_noalloc_f32 holds %zu bytes (use gdn_tm_run_f32)",
                R.L.total, kStaticScratchBytes);
  char* ws = nullptr;
  if ((st = static_scratch(&ws))) return st;
  // The scratch keeps the previous call's contents; prepare() clears all
  // state that the time loop expects to start at zero.
  if ((st = prepare(p, pts, b, ws, R, stream))) return st;
  uint64_t launched = 0;
  for (int base = 0; base < p->n_steps; base += R.L.R)
    launched += enqueue_chunk(R, p, std::min(R.L.R, p->n_steps - base), stream);
  count_launches(launched);
  return finalize(p, b, R, stream);
}

}  // namespace tm2d
}  // namespace gdn

extern "C" int gdn_tm_run_noalloc_f32(const GdnTmParams* p, const GdnTmPoints* pts,
                                      const GdnTmBuffers* b, void* stream) {
  return gdn::tm2d::run_noalloc_f32(p, pts, b, static_cast<cudaStream_t>(stream));
}
