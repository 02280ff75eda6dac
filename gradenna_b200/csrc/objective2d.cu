// The built-in 2D objective w_prad sum_k P_k + w_s11 sum_k |S11_k|^2 and the
// adjoint run's CW source weights, straight from the forward run's DFT
// monitor outputs, in one launch.
//
//   P_k   monitors.py:20-70 (closed dual-grid contour flux, as gdn_poynting_box_2d)
//   V, I  freq_adjoint.py:536-558 (port phasors rebuilt from the fields)
//   S11   sparams.py:68-79 (Kurokawa power wave, real reference resistance)
//   W     freq_adjoint.py:317-352 (cotangent times the Jz / magnetic basis)
//
// One CTA per frequency: a block reduction gives P_k, thread 0 forms S11_k,
// then the CTA writes its column of the weight lists (contour faces in a
// fixed order, with a barrier between faces, so corner cells shared by two
// faces are updated by one thread at a time; deterministic). The CTA that
// finishes last (an atomic ticket, no waiting) sums the per-frequency
// objective terms into the value and re-arms the ticket.
#include <algorithm>
#include <array>
#include <map>

#include "common.cuh"

namespace gdn {
namespace obj2d {

struct Ref {  // a phasor sample: monitor, element offset at k = 0, stride per frequency
  int mon;
  long long off, ks;
};

struct CPt {  // one contour point of the flux
  Ref e0, e1, h;
  int w0, w1, wh;  // rows of e0, e1 in the Ez list and of h in the Hx or Hy list
  int hkind;       // 1 = Hx, 2 = Hy
  double coef;     // flux = coef Re(avg(e0, e1) conj(h))
};

struct PortRefs {
  Ref r[5];  // Ez(i,j), Hy(i,j), Hy(i-1,j), Hx(i,j), Hx(i,j-1)
  int w[5];  // rows in the Ez, Hy, Hy, Hx, Hx lists
};

struct Args {
  int K, n_pts, face_end[4], n_ez, n_hx, n_hy;
  const double2* const* mon;
  const CPt* pts;
  PortRefs port;
  const double2* cv;  // per frequency: V = cv_k E
  double dx, dy, R, w_prad, w_s11, basis_e, basis_h;
  double *partial, *value, *p_rad;
  double2* s11;
  double2 *w_ez, *w_hx, *w_hy;
  unsigned* ticket;
};

__device__ __forceinline__ double2 ld(const Args& a, const Ref& r, int k) {
  return a.mon[r.mon][r.off + (long long)k * r.ks];
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ void cadd(double2* p, double2 v, double s) {
  p->x += s * v.x;
  p->y += s * v.y;
}

__global__ void __launch_bounds__(256) prad_s11_kernel(Args a) {
  const int k = blockIdx.x, K = a.K;
  __shared__ double red[32];
  __shared__ double2 s_port[2];  // g_E at the port's Ez, g_I
  // Flux P_k.
  double acc = 0.0;
  for (int t = threadIdx.x; t < a.n_pts; t += blockDim.x) {
    const CPt& p = a.pts[t];
    const double2 e0 = ld(a, p.e0, k), e1 = ld(a, p.e1, k), h = ld(a, p.h, k);
    acc += p.coef * (0.5 * (e0.x + e1.x) * h.x + 0.5 * (e0.y + e1.y) * h.y);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  // Zero this frequency's column of the weight lists.
  for (int m = threadIdx.x; m < a.n_ez; m += blockDim.x) a.w_ez[(long long)m * K + k] = make_double2(0, 0);
  for (int m = threadIdx.x; m < a.n_hx; m += blockDim.x) a.w_hx[(long long)m * K + k] = make_double2(0, 0);
  for (int m = threadIdx.x; m < a.n_hy; m += blockDim.x) a.w_hy[(long long)m * K + k] = make_double2(0, 0);
  __syncthreads();
  if (threadIdx.x == 0) {
    double P = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) P += red[w];
    // Port phasors and S11 (holomorphic chain: torch's gradient of a real L
    // through s = N / D is g_s conj(ds/dz)).
    const PortRefs& q = a.port;
    const double2 E = ld(a, q.r[0], k);
    const double2 hy1 = ld(a, q.r[1], k), hy0 = ld(a, q.r[2], k);
    const double2 hx1 = ld(a, q.r[3], k), hx0 = ld(a, q.r[4], k);
    const double2 V = cmul(a.cv[k], E);
    const double2 I = make_double2((hy1.x - hy0.x) * a.dy - (hx1.x - hx0.x) * a.dx,
                                   (hy1.y - hy0.y) * a.dy - (hx1.y - hx0.y) * a.dx);
    const double2 N = make_double2(V.x - a.R * I.x, V.y - a.R * I.y);
    const double2 D = make_double2(V.x + a.R * I.x, V.y + a.R * I.y);
    const double2 s = cdiv(N, D);
    a.partial[k] = a.w_prad * P + a.w_s11 * (s.x * s.x + s.y * s.y);
    if (a.p_rad) a.p_rad[k] = P;
    if (a.s11) a.s11[k] = s;
    const double2 gs = make_double2(2.0 * a.w_s11 * s.x, 2.0 * a.w_s11 * s.y);
    const double2 D2 = cmul(D, D);
    const double2 dsdV = cdiv(make_double2(2.0 * a.R * I.x, 2.0 * a.R * I.y), D2);
    const double2 dsdI = cdiv(make_double2(-2.0 * a.R * V.x, -2.0 * a.R * V.y), D2);
    const double2 gV = cmul(gs, cconj(dsdV));
    s_port[0] = cmul(gV, cconj(a.cv[k]));
    s_port[1] = cmul(gs, cconj(dsdI));
  }
  // Flux cotangents, face by face.
  for (int f = 0; f < 4; ++f) {
    const int t0 = f == 0 ? 0 : a.face_end[f - 1], t1 = a.face_end[f];
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
      const CPt& p = a.pts[t];
      const double2 e0 = ld(a, p.e0, k), e1 = ld(a, p.e1, k), h = ld(a, p.h, k);
      const double s = a.w_prad * p.coef;
      cadd(&a.w_ez[(long long)p.w0 * K + k], h, 0.5 * s);
      cadd(&a.w_ez[(long long)p.w1 * K + k], h, 0.5 * s);
      double2* wh = (p.hkind == 1 ? a.w_hx : a.w_hy) + (long long)p.wh * K + k;
      cadd(wh, make_double2(0.5 * (e0.x + e1.x), 0.5 * (e0.y + e1.y)), s);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const PortRefs& q = a.port;
    cadd(&a.w_ez[(long long)q.w[0] * K + k], s_port[0], 1.0);
    cadd(&a.w_hy[(long long)q.w[1] * K + k], s_port[1], a.dy);
    cadd(&a.w_hy[(long long)q.w[2] * K + k], s_port[1], -a.dy);
    cadd(&a.w_hx[(long long)q.w[3] * K + k], s_port[1], -a.dx);
    cadd(&a.w_hx[(long long)q.w[4] * K + k], s_port[1], a.dx);
  }
  __syncthreads();
  // Gradients -> adjoint CW weights: W = conj(g) * basis.
  for (int m = threadIdx.x; m < a.n_ez; m += blockDim.x) {
    double2* p = &a.w_ez[(long long)m * K + k];
    *p = make_double2(p->x * a.basis_e, -p->y * a.basis_e);
  }
  for (int m = threadIdx.x; m < a.n_hx; m += blockDim.x) {
    double2* p = &a.w_hx[(long long)m * K + k];
    *p = make_double2(p->x * a.basis_h, -p->y * a.basis_h);
  }
  for (int m = threadIdx.x; m < a.n_hy; m += blockDim.x) {
    double2* p = &a.w_hy[(long long)m * K + k];
    *p = make_double2(p->x * a.basis_h, -p->y * a.basis_h);
  }
  // The last CTA to finish sums the per-frequency terms.
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(a.ticket, 1u) == unsigned(K - 1);
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double v = 0.0;
    for (int kk = 0; kk < K; ++kk) v += const_cast<volatile double*>(a.partial)[kk];
    *a.value = v;
    *a.ticket = 0u;
  }
}

// Host side: cell lists, phasor references and the contour table.
struct Plan {
  std::vector<std::array<int, 2>> ez, hx, hy;
  std::vector<CPt> pts;
  int face_end[4] = {0, 0, 0, 0};
  PortRefs port{};
};

static int find_ref(const GdnTmObjective* o, int comp, int i, int j, Ref* r) {
  for (int m = 0; m < o->n_monitors; ++m) {
    const GdnDftMonitor& g = o->monitors[m];
    if (g.comp != comp || i < g.lo[0] || i >= g.hi[0] || j < g.lo[1] || j >= g.hi[1]) continue;
    const long long w = g.hi[1] - g.lo[1], h = g.hi[0] - g.lo[0];
    *r = Ref{m, (long long)(i - g.lo[0]) * w + (j - g.lo[1]), h * w};
    return GDN_OK;
  }
  GDN_BAD_ARG("no DFT monitor covers component %d cell (%d, %d) read by the objective", comp, i, j);
}

static int make_plan(const GdnTmObjective* o, Plan* pl, bool refs) {
  if (!o) GDN_BAD_ARG("null objective");
  const int il = o->box[0], ir = o->box[1], jb = o->box[2], jt = o->box[3];
  if (!(0 <= il && il < ir && ir < o->nx - 1 && 0 <= jb && jb < jt && jt < o->ny - 1))
    GDN_BAD_ARG("box (%d, %d, %d, %d) is not a valid contour on a %dx%d grid", il, ir, jb, jt,
                o->nx, o->ny);
  const int pi = o->port[0], pj = o->port[1];
  if (pi < 1 || pj < 1 || pi > o->nx - 2 || pj > o->ny - 2)
    GDN_BAD_ARG("port (%d, %d) outside the valid range (margin 1)", pi, pj);
  std::map<std::array<int, 2>, int> mez, mhx, mhy;
  auto row = [](std::map<std::array<int, 2>, int>& mp, std::vector<std::array<int, 2>>& v, int i,
                int j) {
    auto it = mp.find({i, j});
    if (it != mp.end()) return it->second;
    const int r = int(v.size());
    mp[{i, j}] = r;
    v.push_back({i, j});
    return r;
  };
  int st = GDN_OK;
  auto point = [&](int i0, int j0, int i1, int j1, int hc, int hi, int hj, double coef) {
    CPt p{};
    p.w0 = row(mez, pl->ez, i0, j0);
    p.w1 = row(mez, pl->ez, i1, j1);
    p.hkind = hc;
    p.wh = hc == 1 ? row(mhx, pl->hx, hi, hj) : row(mhy, pl->hy, hi, hj);
    p.coef = coef;
    if (refs && !st) st = find_ref(o, 0, i0, j0, &p.e0);
    if (refs && !st) st = find_ref(o, 0, i1, j1, &p.e1);
    if (refs && !st) st = find_ref(o, hc, hi, hj, &p.h);
    pl->pts.push_back(p);
  };
  for (int j = jb + 1; j <= jt; ++j) point(ir, j, ir + 1, j, 2, ir, j, -0.5 * o->dy);  // right
  pl->face_end[0] = int(pl->pts.size());
  for (int j = jb + 1; j <= jt; ++j) point(il, j, il + 1, j, 2, il, j, 0.5 * o->dy);   // left
  pl->face_end[1] = int(pl->pts.size());
  for (int i = il + 1; i <= ir; ++i) point(i, jt, i, jt + 1, 1, i, jt, 0.5 * o->dx);   // top
  pl->face_end[2] = int(pl->pts.size());
  for (int i = il + 1; i <= ir; ++i) point(i, jb, i, jb + 1, 1, i, jb, -0.5 * o->dx);  // bottom
  pl->face_end[3] = int(pl->pts.size());
  if (st) return st;
  PortRefs& q = pl->port;
  q.w[0] = row(mez, pl->ez, pi, pj);
  q.w[1] = row(mhy, pl->hy, pi, pj);
  q.w[2] = row(mhy, pl->hy, pi - 1, pj);
  q.w[3] = row(mhx, pl->hx, pi, pj);
  q.w[4] = row(mhx, pl->hx, pi, pj - 1);
  if (refs) {
    const int comp[5] = {0, 2, 2, 1, 1};
    const int ci[5] = {pi, pi, pi - 1, pi, pi}, cj[5] = {pj, pj, pj, pj, pj - 1};
    for (int t = 0; t < 5; ++t)
      if ((st = find_ref(o, comp[t], ci[t], cj[t], &q.r[t]))) return st;
  }
  return GDN_OK;
}

}  // namespace obj2d
}  // namespace gdn

using namespace gdn::obj2d;

extern "C" int gdn_tm_objective_cells(const GdnTmObjective* o, int32_t* n_ez, int32_t* n_hx,
                                      int32_t* n_hy, int32_t* ez_ij, int32_t* hx_ij,
                                      int32_t* hy_ij) {
  Plan pl;
  int st = make_plan(o, &pl, false);
  if (st) return st;
  if (n_ez) *n_ez = int32_t(pl.ez.size());
  if (n_hx) *n_hx = int32_t(pl.hx.size());
  if (n_hy) *n_hy = int32_t(pl.hy.size());
  const std::vector<std::array<int, 2>>* lists[3] = {&pl.ez, &pl.hx, &pl.hy};
  int32_t* outs[3] = {ez_ij, hx_ij, hy_ij};
  for (int t = 0; t < 3; ++t)
    if (outs[t])
      for (size_t m = 0; m < lists[t]->size(); ++m) {
        outs[t][2 * m] = (*lists[t])[m][0];
        outs[t][2 * m + 1] = (*lists[t])[m][1];
      }
  return GDN_OK;
}

extern "C" int gdn_tm_objective_prad_s11(const GdnTmObjective* o, void* stream) {
  Plan pl;
  int st = make_plan(o, &pl, true);
  if (st) return st;
  const int K = o->n_freq;
  if (K <= 0 || !o->freqs) GDN_BAD_ARG("need n_freq > 0 and the frequencies");
  if (!o->value || !o->w_ez || !o->w_hx || !o->w_hy) GDN_BAD_ARG("null output");
  for (int m = 0; m < o->n_monitors; ++m)
    if (!o->monitors[m].out) GDN_BAD_ARG("monitor %d: output is null", m);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // V_k = cv_k E: -dz (E / z + E) / 2 * z^(1/2), z = exp(i w dt).
  std::vector<double2> cv(K);
  for (int k = 0; k < K; ++k) {
    const double om = 2.0 * 3.14159265358979323846 * o->freqs[k] * o->dt;
    const double zr = cos(om), zi = sin(om), hr = cos(0.5 * om), hi = sin(0.5 * om);
    // 1/z + 1 = conj(z) + 1 (|z| = 1)
    const double ar = zr + 1.0, ai = -zi;
    cv[k] = make_double2(-o->dz * 0.5 * (ar * hr - ai * hi), -o->dz * 0.5 * (ar * hi + ai * hr));
  }
  std::vector<const double2*> mons(std::max(o->n_monitors, 1), nullptr);
  for (int m = 0; m < o->n_monitors; ++m) mons[m] = static_cast<const double2*>(o->monitors[m].out);
  gdn::Carve cv_;
  const size_t o_mon = cv_.take<const double2*>(mons.size());
  const size_t o_pts = cv_.take<CPt>(std::max<size_t>(pl.pts.size(), 1));
  const size_t o_cv = cv_.take<double2>(K);
  const size_t o_part = cv_.take<double>(K);
  const size_t o_tick = cv_.take<unsigned>(1);
  char* ws = nullptr;
  GDN_TRY_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ws), cv_.bytes(), s));
  struct Guard {
    char* p;
    cudaStream_t s;
    ~Guard() { cudaFreeAsync(p, s); }
  } guard{ws, s};
  GDN_TRY_CUDA(cudaMemcpyAsync(ws + o_mon, mons.data(), mons.size() * sizeof(void*),
                               cudaMemcpyHostToDevice, s));
  if (!pl.pts.empty())
    GDN_TRY_CUDA(cudaMemcpyAsync(ws + o_pts, pl.pts.data(), pl.pts.size() * sizeof(CPt),
                                 cudaMemcpyHostToDevice, s));
  GDN_TRY_CUDA(cudaMemcpyAsync(ws + o_cv, cv.data(), K * sizeof(double2), cudaMemcpyHostToDevice, s));
  GDN_TRY_CUDA(cudaMemsetAsync(ws + o_tick, 0, sizeof(unsigned), s));
  Args a{};
  a.K = K;
  a.n_pts = int(pl.pts.size());
  for (int f = 0; f < 4; ++f) a.face_end[f] = pl.face_end[f];
  a.n_ez = int(pl.ez.size());
  a.n_hx = int(pl.hx.size());
  a.n_hy = int(pl.hy.size());
  a.mon = reinterpret_cast<const double2* const*>(ws + o_mon);
  a.pts = reinterpret_cast<const CPt*>(ws + o_pts);
  a.port = pl.port;
  a.cv = reinterpret_cast<const double2*>(ws + o_cv);
  a.dx = o->dx;
  a.dy = o->dy;
  a.R = o->resistance;
  a.w_prad = o->w_prad;
  a.w_s11 = o->w_s11;
  a.basis_e = 1.0 / (-((o->dt / o->eps0) / (o->dx * o->dy)));
  a.basis_h = (-o->eps0 / o->mu0) / (-(o->dt / o->mu0));
  a.partial = reinterpret_cast<double*>(ws + o_part);
  a.value = o->value;
  a.p_rad = o->p_rad;
  a.s11 = static_cast<double2*>(o->s11);
  a.w_ez = static_cast<double2*>(o->w_ez);
  a.w_hx = static_cast<double2*>(o->w_hx);
  a.w_hy = static_cast<double2*>(o->w_hy);
  a.ticket = reinterpret_cast<unsigned*>(ws + o_tick);
  prad_s11_kernel<<<K, 256, 0, s>>>(a);
  gdn::count_launches(1);
  GDN_TRY_CUDA(cudaGetLastError());
  return GDN_OK;
}
