// 2D TM time loop, register-resident row march (included by tm2d.cu inside
// namespace gdn::tm2d).
//
// Same per-step semantics as tb_body (fdtd2d.py:412-464: H with CPML psi ->
// Mx/My -> port current + Ez^n snapshot -> E with psi -> Jz -> RVS ports and
// V -> probes; monitor-ring writes for the running DFT), organised so that
// the field state never goes through shared memory:
//
//   * A warp owns a strip of 32*V columns (V cells per lane, one 8-byte
//     vector) and marches down a segment of rows. Its owned columns are the
//     middle 32*V - 2*HJ; the HJ = 4 columns on each side are a halo that the
//     neighbouring strips own. Owned rows are [i0, i0 + rows); the march
//     reads TB rows above and below.
//   * One launch advances TB = 4 time steps as a wavefront: at march step t
//     row t is loaded and level s (time step n0 + s - 1) updates row t - s,
//     so level s sees level s-1's new row below it and its own previous row
//     above it. Rows in flight sit in a register shift register: slot s holds
//     row t - s, level s updates slot s in place, row t - TB leaves as a
//     finished row after level TB, and the slots move down by one per step
//     (register moves keep the loop body one step long, small enough for the
//     instruction cache with many warps per SM).
//   * Horizontal neighbours come from warp shuffles (Ez to the right for H,
//     Hx to the left for E); vertical neighbours are the adjacent slots.
//     Wrong values at the strip's outer lanes stay inside the halo: each
//     level spoils one more column per side, HJ >= TB.
//   * Rows arrive through a per-warp cp.async ring PF rows ahead of use.
//     Warps are independent: no block-wide barrier anywhere.
//   * Point work (sources, ports, probes, magnetic currents) is one list per
//     warp sorted by row; a level looks at it only on rows that hold points,
//     and those rows go through a small shared-memory row scratch handled by
//     out-of-line code. Injections apply to every copy of a cell, records come
//     from the owner.
//   * Template flags: XS = the strip segment touches an x CPML slab or the
//     x PEC rows (row masks, ezx/hyx psi, row coefficients staged in shared
//     memory); YS = likewise for y (column masks and coefficients in
//     registers, ezy/hxy psi). Interior warps (neither) run the bare stencil.
#pragma once

namespace march {

constexpr int TB = 4;         // time steps per launch (levels of the wavefront)
constexpr int NSL = TB + 2;   // register row slots: rows t .. t - TB - 1
constexpr int PF = 3;         // rows requested ahead of use
constexpr int NST = PF + 2;   // cp.async ring stages per warp (one spare: no reuse hazard)
constexpr int WPB = 4;        // warps per CTA
constexpr int HJ = 4;         // halo columns per side (>= TB, a multiple of V)
constexpr int SIMAX = 64;     // most owned rows per segment
constexpr int MAXE = 256;     // point entries per warp whose values are staged
constexpr int MAXMW = 8;      // monitor parts per warp staged in shared memory

// Point entry types, in the order a step processes them.
enum : int { P_MX = 0, P_MY = 1, P_PORT = 2, P_SRC = 3, P_PROBE = 4 };

template <typename T>
struct Lanes;
template <>
struct Lanes<float> {
  static constexpr int V = 2;  // 8-byte vectors
};
template <>
struct Lanes<double> {
  static constexpr int V = 1;
};

template <typename T>
__host__ __device__ constexpr int owned_cols() {
  return 32 * Lanes<T>::V - 2 * HJ;
}

template <typename T, bool XS, bool YS>
__host__ __device__ constexpr int planes() {
  return 5 + (XS ? 2 : 0) + (YS ? 2 : 0);
}

// Shared-memory bytes per warp (every part a multiple of 16 bytes): the
// cp.async ring, staged point values, x-slab row coefficients, monitor parts
// and the 5-row point scratch.
template <typename T, bool XS, bool YS>
__host__ __device__ constexpr size_t warp_smem() {
  return size_t(NST) * planes<T, XS, YS>() * 32 * Lanes<T>::V * sizeof(T) +
         size_t(MAXE) * TB * sizeof(T) + (XS ? size_t(SIMAX + 2 * TB) * 8 * sizeof(T) : 0) +
         size_t(MAXMW) * sizeof(MonW) + size_t(5) * 32 * Lanes<T>::V * sizeof(T);
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Value of a staged-or-computed point term for entry e (index in the warp's
// list), type ty, point m, sub-step s, absolute step n.
template <typename T>
__device__ __forceinline__ T entry_value(const Dev<T>& d, const T* sval, int e, int ty, int m,
                                         int s, int n) {
  if (e < MAXE) return sval[e * TB + s];
  switch (ty) {
    case P_MX: return mx_term(d, m, n);
    case P_MY: return my_term(d, m, n);
    case P_SRC: return src_term(d, m, n);
    default: return d.cb_vs[m] * d.port_vs[(long long)n * d.n_ports + m];
  }
}

// Point work of one row on the warp's row scratch `row` = [E^n | Hx | Hy |
// Hy of the row above | E^{n+1}], 32*V columns each starting at column je.
// The row's entries are spread over the lanes; injections are shared-memory
// atomic adds, so several entries on one cell all land. Returns the end of
// the row's entries (they are a prefix of [q0, pe): the list is sorted by
// row and q0 is the first entry of row r).
template <typename T>
__device__ __noinline__ int points_h(const Dev<T>& d, int pb, int pe, const T* sval, T* row,
                                     int je, int q0, int r, int s, int n) {
  constexpr int RW = 32 * Lanes<T>::V;
  const int lane = threadIdx.x & 31;
  int q1 = q0;
  for (;;) {
    const int q = q1 + lane;
    const unsigned in = __ballot_sync(0xffffffffu, q < pe && d.mpts[q].i == r);
    q1 += __popc(in);
    if (in != 0xffffffffu) break;
  }
  for (int q = q0 + lane; q < q1; q += 32) {  // Mx / My (fdtd2d.py:419-428)
    const MPt p = d.mpts[q];
    const int ty = p.tag & 7;
    if (ty == P_MX || ty == P_MY)
      atomicAdd(row + (ty == P_MX ? RW : 2 * RW) + (p.j - je),
                -entry_value(d, sval, q - pb, ty, p.m, s, n));
  }
  __syncwarp();
  for (int q = q0 + lane; q < q1; q += 32) {  // port current on H^{n+1/2} (fdtd2d.py:430-436)
    const MPt p = d.mpts[q];
    const int o = p.j - je;
    if ((p.tag & 7) == P_PORT && (p.tag & 8))
      d.out_i[(long long)n * d.n_ports + p.m] =
          (row[2 * RW + o] - row[3 * RW + o]) * d.dy - (row[RW + o] - row[RW + o - 1]) * d.dx;
  }
  return q1;
}

template <typename T>
__device__ __noinline__ void points_e(const Dev<T>& d, int pb, const T* sval, T* row, int je,
                                      int q0, int q1, int s, int n) {
  constexpr int RW = 32 * Lanes<T>::V;
  const int lane = threadIdx.x & 31;
  T* en = row + 4 * RW;
  for (int q = q0 + lane; q < q1; q += 32) {  // Jz (fdtd2d.py:444)
    const MPt p = d.mpts[q];
    if ((p.tag & 7) == P_SRC)
      atomicAdd(en + (p.j - je), -entry_value(d, sval, q - pb, P_SRC, p.m, s, n));
  }
  __syncwarp();
  for (int q = q0 + lane; q < q1; q += 32) {  // RVS injection, every port (fdtd2d.py:446-448)
    const MPt p = d.mpts[q];
    if ((p.tag & 7) == P_PORT)
      atomicAdd(en + (p.j - je), -entry_value(d, sval, q - pb, P_PORT, p.m, s, n));
  }
  __syncwarp();
  for (int q = q0 + lane; q < q1; q += 32) {  // V (fdtd2d.py:449-451) and probes (:461)
    const MPt p = d.mpts[q];
    const int o = p.j - je, ty = p.tag & 7;
    if (ty == P_PORT && (p.tag & 8))
      d.out_v[(long long)n * d.n_ports + p.m] = T(-0.5) * d.dz * (row[o] + en[o]);
    else if (ty == P_PROBE)
      d.out_probe[(long long)n * d.n_probes + p.m] = en[o];
  }
}

template <typename T, bool XS, bool YS>
struct March {
  static constexpr int V = Lanes<T>::V;
  static constexpr int NPL = planes<T, XS, YS>();
  static constexpr int RW = 32 * V;  // elements of one plane row in a ring stage
  static constexpr bool GEN = XS || YS;

  // Everything the march loop reads is held here by value (registers):
  // reaching the kernel parameters or the task through a reference inside
  // the loop costs a memory load per use.
  const Dev<T>* dp;  // the kernel's parameter block (rare paths only)
  int lane, jl, tstart, nsteps, n0, nsub, par;
  int nx, ld, rend, pb, pe, mb, R;
  long long plane, mon_cells;
  T dt_mu, inv_dx, inv_dy;
  const T *src, *ca, *cb, *psrc;
  T *dst, *pdst, *mring;
  const MPt* mpts;
  T *ring, *sval, *rco, *prow;
  const MonW* smw;
  int nmw;

  // Row slots.
  T E[NSL][V], HX[NSL][V], HY[NSL][V], CA[NSL][V], CB[NSL][V];
  T PEX[XS ? NSL : 1][V], PHY[XS ? NSL : 1][V];  // psi ezx, hyx
  T PEY[YS ? NSL : 1][V], PHX[YS ? NSL : 1][V];  // psi ezy, hxy
  // Column data of this lane.
  T cbh[YS ? V : 1], cch[YS ? V : 1], ckh[YS ? V : 1], cbe[YS ? V : 1], cce[YS ? V : 1],
      cke[YS ? V : 1];
  bool cHx[V], cHy[V], cE[V], cown[V];
  // Point cursors, one per level.
  int cur[TB + 1], nextrow[TB + 1];

  __device__ __forceinline__ March(const Dev<T>* d_) : dp(d_) {}

  __device__ __forceinline__ void issue(int i, int st) {
    const long long g = cell_at(ld, i, jl);
    T* s = ring + st * NPL * RW + lane * V;
    cp_async8(s, src + g);
    cp_async8(s + RW, src + plane + g);
    cp_async8(s + 2 * RW, src + 2 * plane + g);
    cp_async8(s + 3 * RW, ca + g);
    cp_async8(s + 4 * RW, cb + g);
    int p = 5;
    if constexpr (XS) {
      cp_async8(s + p * RW, psrc + g);                    // ezx
      cp_async8(s + (p + 1) * RW, psrc + 2 * plane + g);  // hyx
      p += 2;
    }
    if constexpr (YS) {
      cp_async8(s + p * RW, psrc + plane + g);            // ezy
      cp_async8(s + (p + 1) * RW, psrc + 3 * plane + g);  // hxy
    }
  }

  template <int U>
  __device__ __forceinline__ void take(int st) {
    const T* s = ring + st * NPL * RW + lane * V;
#pragma unroll
    for (int c = 0; c < V; ++c) {
      E[U][c] = s[c];
      HX[U][c] = s[RW + c];
      HY[U][c] = s[2 * RW + c];
      CA[U][c] = s[3 * RW + c];
      CB[U][c] = s[4 * RW + c];
    }
    int p = 5;
    if constexpr (XS) {
#pragma unroll
      for (int c = 0; c < V; ++c) {
        PEX[U][c] = s[p * RW + c];
        PHY[U][c] = s[(p + 1) * RW + c];
      }
      p += 2;
    }
    if constexpr (YS) {
#pragma unroll
      for (int c = 0; c < V; ++c) {
        PEY[U][c] = s[p * RW + c];
        PHX[U][c] = s[(p + 1) * RW + c];
      }
    }
  }

  // Level S (time step n0 + S - 1) on the row in slot Q = S; the row below
  // is in slot S - 1 (already at level S - 1), the row above in slot S + 1
  // (at level S since the previous step).
  template <int S>
  __device__ __forceinline__ void level(int r) {
    constexpr int Q = S, QD = S - 1, QU = S + 1;
    const int s = S - 1;
    const int n = n0 + s;
    T* e = E[Q];
    T* hx = HX[Q];
    T* hy = HY[Q];
    const T* edn = E[QD];
    const T* hyu = HY[QU];
    // Row coefficients and masks (x slabs, PEC rows).
    T rbh = 0, rch = 0, rkh = 1, rbe = 0, rce = 0, rke = 1;
    bool rHx = true, rHy = true, rE = true;
    if constexpr (XS) {
      const T* rc = rco + (r - tstart) * 8;
      rbh = rc[0]; rch = rc[1]; rkh = rc[2]; rbe = rc[3]; rce = rc[4]; rke = rc[5];
      rHx = r >= 0 && r < nx;
      rHy = r >= 0 && r < nx - 1;
      rE = r >= 1 && r <= nx - 2;
    }
    // ---- H (fdtd2d.py:416-428) ----
    const T e0r = __shfl_down_sync(0xffffffffu, e[0], 1);
#pragma unroll
    for (int c = 0; c < V; ++c) {
      const T er = c + 1 < V ? e[(c + 1) % V] : e0r;
      const T dEy = (er - e[c]) * inv_dy;
      T thx = dEy;
      if constexpr (YS) {
        PHX[Q][c] = cbh[c] * PHX[Q][c] + cch[c] * dEy;
        thx = dEy * ckh[c] + PHX[Q][c];
      }
      const T dEx = (edn[c] - e[c]) * inv_dx;
      T thy = dEx;
      if constexpr (XS) {
        PHY[Q][c] = rbh * PHY[Q][c] + rch * dEx;
        thy = dEx * rkh + PHY[Q][c];
      }
      if constexpr (GEN) {
        if (rHx && cHx[c]) hx[c] -= dt_mu * thx;
        if (rHy && cHy[c]) hy[c] += dt_mu * thy;
      } else {
        hx[c] -= dt_mu * thx;
        hy[c] += dt_mu * thy;
      }
    }
    // ---- points of this row (fdtd2d.py:419-436, 444-451, 461) ----
    // Rows with points go through the warp's row scratch in shared memory:
    // out-of-line code applies Mx/My and records the port currents on it,
    // the E update runs in registers, then Jz, the RVS injections, V and the
    // probes are applied to the scratch and the row is read back.
    const bool pts = nextrow[S] == r;
    int pend = 0;
    if (pts) {
#pragma unroll
      for (int c = 0; c < V; ++c) {
        prow[lane * V + c] = e[c];
        prow[RW + lane * V + c] = hx[c];
        prow[2 * RW + lane * V + c] = hy[c];
        prow[3 * RW + lane * V + c] = hyu[c];
      }
      __syncwarp();
      pend = points_h<T>(*dp, pb, pe, sval, prow, jl - lane * V, cur[S], r, s, n);
      __syncwarp();
#pragma unroll
      for (int c = 0; c < V; ++c) {
        hx[c] = prow[RW + lane * V + c];
        hy[c] = prow[2 * RW + lane * V + c];
      }
    }
    const T hxl0 = __shfl_up_sync(0xffffffffu, hx[V - 1], 1);
    // ---- E (fdtd2d.py:438-443) ----
#pragma unroll
    for (int c = 0; c < V; ++c) {
      const T hl = c > 0 ? hx[c > 0 ? c - 1 : 0] : hxl0;
      const T dhy = (hy[c] - hyu[c]) * inv_dx;
      const T dhx = (hx[c] - hl) * inv_dy;
      T tx = dhy, ty = dhx;
      if constexpr (XS) {
        PEX[Q][c] = rbe * PEX[Q][c] + rce * dhy;
        tx = dhy * rke + PEX[Q][c];
      }
      if constexpr (YS) {
        PEY[Q][c] = cbe[c] * PEY[Q][c] + cce[c] * dhx;
        ty = dhx * cke[c] + PEY[Q][c];
      }
      if constexpr (GEN) {
        if (rE && cE[c]) e[c] = CA[Q][c] * e[c] + CB[Q][c] * (tx - ty);
      } else {
        e[c] = CA[Q][c] * e[c] + CB[Q][c] * (tx - ty);
      }
    }
    if (pts) {
#pragma unroll
      for (int c = 0; c < V; ++c) prow[4 * RW + lane * V + c] = e[c];
      __syncwarp();
      points_e<T>(*dp, pb, sval, prow, jl - lane * V, cur[S], pend, s, n);
      __syncwarp();
#pragma unroll
      for (int c = 0; c < V; ++c) e[c] = prow[4 * RW + lane * V + c];
      cur[S] = pend;
      nextrow[S] = pend < pe ? mpts[pend].i : 0x7fffffff;
    }
    // ---- monitor ring (running DFT, fdtd2d.py:453-458) ----
    if (nmw > 0) {
      T* slot = mring + (long long)(n % R) * mon_cells;
      for (int q = 0; q < nmw; ++q) {
        const MonW w = q < MAXMW ? smw[q] : dp->mw[mb + q];
        if (r < w.a0 || r >= w.a1) continue;
        T* o = slot + w.base + (long long)r * w.w;
#pragma unroll
        for (int c = 0; c < V; ++c) {
          const int j = jl + c;
          if (j >= w.b0 && j < w.b1) o[j] = w.comp == 0 ? e[c] : (w.comp == 1 ? hx[c] : hy[c]);
        }
      }
    }
  }

  // The finished row in slot Q (level TB) to the other state slot.
  template <int Q>
  __device__ __forceinline__ void store(int r) {
    const long long g = cell_at(ld, r, jl);
    T* pd = pdst;
    if constexpr (V == 2) {
      if (cown[0] && cown[1]) {
        using V2 = typename std::conditional<sizeof(T) == 4, float2, double2>::type;
        *reinterpret_cast<V2*>(dst + g) = V2{E[Q][0], E[Q][1]};
        *reinterpret_cast<V2*>(dst + plane + g) = V2{HX[Q][0], HX[Q][1]};
        *reinterpret_cast<V2*>(dst + 2 * plane + g) = V2{HY[Q][0], HY[Q][1]};
        if constexpr (XS) {
          *reinterpret_cast<V2*>(pd + g) = V2{PEX[Q][0], PEX[Q][1]};
          *reinterpret_cast<V2*>(pd + 2 * plane + g) = V2{PHY[Q][0], PHY[Q][1]};
        }
        if constexpr (YS) {
          *reinterpret_cast<V2*>(pd + plane + g) = V2{PEY[Q][0], PEY[Q][1]};
          *reinterpret_cast<V2*>(pd + 3 * plane + g) = V2{PHX[Q][0], PHX[Q][1]};
        }
        return;
      }
    }
#pragma unroll
    for (int c = 0; c < V; ++c) {
      if (!cown[c]) continue;
      dst[g + c] = E[Q][c];
      dst[plane + g + c] = HX[Q][c];
      dst[2 * plane + g + c] = HY[Q][c];
      if constexpr (XS) {
        pd[g + c] = PEX[Q][c];
        pd[2 * plane + g + c] = PHY[Q][c];
      }
      if constexpr (YS) {
        pd[plane + g + c] = PEY[Q][c];
        pd[3 * plane + g + c] = PHX[Q][c];
      }
    }
  }

  // Move every slot down by one row; the last slot keeps only Hy (the row
  // above level TB).
  __device__ __forceinline__ void shift() {
#pragma unroll
    for (int c = 0; c < V; ++c) HY[TB + 1][c] = HY[TB][c];
#pragma unroll
    for (int u = TB; u >= 1; --u)
#pragma unroll
      for (int c = 0; c < V; ++c) {
        E[u][c] = E[u - 1][c];
        HX[u][c] = HX[u - 1][c];
        HY[u][c] = HY[u - 1][c];
        CA[u][c] = CA[u - 1][c];
        CB[u][c] = CB[u - 1][c];
        if constexpr (XS) {
          PEX[u][c] = PEX[u - 1][c];
          PHY[u][c] = PHY[u - 1][c];
        }
        if constexpr (YS) {
          PEY[u][c] = PEY[u - 1][c];
          PHX[u][c] = PHX[u - 1][c];
        }
      }
  }

  // March step k: row t = tstart + k enters slot 0.
  __device__ __forceinline__ void step(int k) {
    cp_async_wait<PF - 1>();
    take<0>(k % NST);
    if (k + PF < nsteps) issue(tstart + k + PF, (k + PF) % NST);
    cp_async_commit();
    const int t = tstart + k;
    static_assert(TB == 4, "levels are unrolled for TB = 4");
    if (k >= 1 && nsub >= 1) level<1>(t - 1);
    if (k >= 2 && nsub >= 2) level<2>(t - 2);
    if (k >= 3 && nsub >= 3) level<3>(t - 3);
    if (k >= 4 && nsub >= 4) level<4>(t - 4);
    const int r = t - TB;
    if (k >= 2 * TB && r < rend) store<TB>(r);
    shift();
  }
};

template <typename T, bool XS, bool YS>
__global__ void __launch_bounds__(WPB * 32) tm_march(const __grid_constant__ Dev<T> d,
                                                      const MTask* tasks, int ntask, int sub0,
                                                      int nsub) {
  constexpr int V = Lanes<T>::V;
  const int warp = threadIdx.x >> 5;
  const int tix = blockIdx.x * WPB + warp;
  if (tix >= ntask) return;  // whole warps only; no block-wide barrier follows
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* wsm = smem_raw + size_t(warp) * warp_smem<T, XS, YS>();
  const MTask tk = tasks[tix];
  March<T, XS, YS> m(&d);
  m.lane = threadIdx.x & 31;
  m.ring = reinterpret_cast<T*>(wsm);
  m.sval = m.ring + NST * planes<T, XS, YS>() * 32 * V;
  m.rco = m.sval + MAXE * TB;
  MonW* smw = reinterpret_cast<MonW*>(m.rco + (XS ? (SIMAX + 2 * TB) * 8 : 0));
  m.smw = smw;
  m.prow = reinterpret_cast<T*>(smw + MAXMW);
  m.n0 = *d.step_base + sub0;
  m.nsub = nsub;
  m.par = (m.n0 / TB) & 1;
  m.jl = tk.j0 - HJ + m.lane * V;
  m.tstart = tk.i0 - TB;
  m.nsteps = tk.rows + 2 * TB;
  m.nx = d.nx;
  m.ld = d.ld;
  m.rend = min(tk.i0 + tk.rows, d.nx);
  m.pb = tk.pb;
  m.pe = tk.pe;
  m.mb = tk.mb;
  m.R = d.R;
  m.plane = d.plane;
  m.mon_cells = d.mon_cells;
  m.dt_mu = d.dt_mu;
  m.inv_dx = d.inv_dx;
  m.inv_dy = d.inv_dy;
  m.src = d.state[m.par];
  m.dst = d.state[m.par ^ 1];
  m.ca = d.ca;
  m.cb = d.cb;
  m.psrc = d.psi[m.par];
  m.pdst = d.psi[m.par ^ 1];
  m.mring = d.mring;
  m.mpts = d.mpts;
  const int lane = m.lane;
  // Start the ring first so the copies overlap the set-up below.
#pragma unroll
  for (int p = 0; p < PF; ++p) {
    if (p < m.nsteps) m.issue(m.tstart + p, p);
    cp_async_commit();
  }
  // Column masks / ownership and y-slab coefficients of this lane.
  const int nx = d.nx, ny = d.ny, npml = d.npml;
#pragma unroll
  for (int c = 0; c < V; ++c) {
    const int j = m.jl + c;
    m.cHx[c] = j >= 0 && j < ny - 1;
    m.cHy[c] = j >= 0 && j < ny;
    m.cE[c] = j >= 1 && j <= ny - 2;
    m.cown[c] = j >= tk.j0 && j < tk.j0 + owned_cols<T>() && j < ny;
    if constexpr (YS) {
      T b = 0, cc = 0, kk = 1;
      if (j >= 0 && j < ny - 1) {
        if (j < npml) {
          b = d.b_hxy_lo[j]; cc = d.c_hxy_lo[j]; kk = d.iky_h[j];
        } else if (j >= ny - 1 - npml) {
          b = d.b_hxy_hi[j - (ny - 1 - npml)]; cc = d.c_hxy_hi[j - (ny - 1 - npml)]; kk = d.iky_h[j];
        }
      }
      m.cbh[c] = b; m.cch[c] = cc; m.ckh[c] = kk;
      const int bb = j - 1, nj = ny - 2;
      b = 0; cc = 0; kk = 1;
      if (bb >= 0 && bb < nj) {
        if (bb < npml) {
          b = d.b_ezy_lo[bb]; cc = d.c_ezy_lo[bb]; kk = d.iky_e[bb];
        } else if (bb >= nj - npml) {
          b = d.b_ezy_hi[bb - (nj - npml)]; cc = d.c_ezy_hi[bb - (nj - npml)]; kk = d.iky_e[bb];
        }
      }
      m.cbe[c] = b; m.cce[c] = cc; m.cke[c] = kk;
    }
  }
  // Row coefficients of the x slabs for every row the march touches.
  if constexpr (XS) {
    for (int q = lane; q < m.nsteps; q += 32) {
      const int i = m.tstart + q;
      T* rc = m.rco + q * 8;
      T b = 0, cc = 0, kk = 1;
      if (i >= 0 && i < nx - 1) {
        if (i < npml) {
          b = d.b_hyx_lo[i]; cc = d.c_hyx_lo[i]; kk = d.ikx_h[i];
        } else if (i >= nx - 1 - npml) {
          b = d.b_hyx_hi[i - (nx - 1 - npml)]; cc = d.c_hyx_hi[i - (nx - 1 - npml)]; kk = d.ikx_h[i];
        }
      }
      rc[0] = b; rc[1] = cc; rc[2] = kk;
      const int a = i - 1, ni = nx - 2;
      b = 0; cc = 0; kk = 1;
      if (a >= 0 && a < ni) {
        if (a < npml) {
          b = d.b_ezx_lo[a]; cc = d.c_ezx_lo[a]; kk = d.ikx_e[a];
        } else if (a >= ni - npml) {
          b = d.b_ezx_hi[a - (ni - npml)]; cc = d.c_ezx_hi[a - (ni - npml)]; kk = d.ikx_e[a];
        }
      }
      rc[3] = b; rc[4] = cc; rc[5] = kk;
    }
  }
  // Point values of this launch's sub-steps and the monitor parts.
  const int np = tk.pe - tk.pb;
  for (int q = lane; q < min(np, MAXE) * TB; q += 32) {
    const int e = q / TB, s = q - e * TB;
    if (s >= nsub) continue;
    const MPt p = d.mpts[tk.pb + e];
    const int ty = p.tag & 7, n = m.n0 + s;
    T v = 0;
    if (ty == P_MX) v = mx_term(d, p.m, n);
    else if (ty == P_MY) v = my_term(d, p.m, n);
    else if (ty == P_SRC) v = src_term(d, p.m, n);
    else if (ty == P_PORT) v = d.cb_vs[p.m] * d.port_vs[(long long)n * d.n_ports + p.m];
    m.sval[q] = v;
  }
  m.nmw = tk.me - tk.mb;
  for (int q = lane; q < min(m.nmw, MAXMW); q += 32) smw[q] = d.mw[tk.mb + q];
#pragma unroll
  for (int s = 0; s <= TB; ++s) {
    m.cur[s] = tk.pb;
    m.nextrow[s] = np > 0 ? d.mpts[tk.pb].i : 0x7fffffff;
  }
#pragma unroll
  for (int u = 0; u < NSL; ++u)
#pragma unroll
    for (int c = 0; c < V; ++c) {
      m.E[u][c] = m.HX[u][c] = m.HY[u][c] = m.CA[u][c] = m.CB[u][c] = T(0);
      if constexpr (XS) m.PEX[u][c] = m.PHY[u][c] = T(0);
      if constexpr (YS) m.PEY[u][c] = m.PHX[u][c] = T(0);
    }
  __syncwarp();
  for (int k = 0; k < m.nsteps; ++k) m.step(k);
  cp_async_wait<0>();
}

}  // namespace march
