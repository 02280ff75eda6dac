/*
 * gradenna_b200 -- C ABI of the B200 (sm_100a) FDTD time-stepping library.
 *
 * This header is the drop-in boundary that replaces the reference's native
 * FFI for the FDTD hot path:
 *
 *   reference symbol                              replaced by
 *   ------------------------------------------------------------------------
 *   gradenna_tm_run_f32 / _f64                    gdn_tm_run_f32 / _f64
 *     (rust/src/lib.rs:89-142, bound in src/gradenna/native.py:140-170)
 *   gradenna_3d_run_f32 / _f64                    gdn_yee_run_f32 / _f64
 *     (rust/src/lib3d.rs:191-230, bound in src/gradenna/native3d.py:145-163)
 *   simulate_tm_native / simulate_3d_native       the Python shim
 *     (src/gradenna/native.py:200, native3d.py:174) gradenna_b200.simulate_tm
 *
 * Conventions (all entry points):
 *   - Every entry point returns a GdnStatus (0 = success) and never aborts;
 *     gdn_last_error() gives a one-line message for the calling thread.
 *     (The reference Rust kernels return void and abort on panic.)
 *   - Bulk arrays (coefficient tables, waveforms, outputs, workspace) are
 *     DEVICE pointers on the current CUDA device. The small index lists in the
 *     *Points structs are HOST pointers (they are binned by tile on the host).
 *   - Arrays are C-order (last axis contiguous) with the reference's shapes:
 *     ez (nx, ny), hx (nx, ny-1), hy (nx-1, ny); waveforms (n_steps, n).
 *   - Complex DFT outputs are interleaved (re, im) pairs, float (complex64)
 *     or double (complex128) as selected by dft_f64, shape (n_freq, ...).
 *     Output DFT buffers are written, not accumulated into: the library zeroes
 *     them. (The reference required caller-zeroed outputs: native.py:409-423.)
 *   - Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default)
 *     and the call returns without synchronising, except where a status must
 *     be read back (documented per entry point).
 *   - The caller owns every buffer. Scratch: pass `workspace` of at least
 *     gdn_*_workspace_size() bytes, or NULL to let the library allocate it
 *     stream-ordered for the duration of the call.
 */
#ifndef GRADENNA_B200_H
#define GRADENNA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum GdnStatus {
  GDN_OK = 0,
  GDN_ERR_BAD_ARG = 1,     /* invalid sizes, indices or null pointers         */
  GDN_ERR_OOM = 2,         /* device allocation failed                          */
  GDN_ERR_CUDA = 3,        /* a CUDA runtime call failed                        */
  GDN_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up                */
  GDN_ERR_NONFINITE = 5,   /* a NaN/Inf was detected where it is checked       */
  GDN_ERR_UNSUPPORTED = 6  /* requested feature not built for this device       */
} GdnStatus;

/* Library version string, e.g. "gradenna_b200 0.1 (sm_100a)". */
const char* gdn_version(void);

/* Message describing the last non-zero status returned on this thread. */
const char* gdn_last_error(void);

/* Number of this library's CUDA kernels launched so far in this process
 * (graph replays count every kernel node they run). No reference
 * counterpart: it lets callers and benchmarks attribute device work. */
uint64_t gdn_kernel_launches(void);

/* Device time of the time loops run since the last reset. Every
 * gdn_tm_run_f32/f64 and gdn_yee_run_f32/f64 records CUDA events on its
 * stream around the replay of its time loop (the step kernels, DFT folds and
 * step-counter advances); this call waits for those events and returns the
 * summed milliseconds, the summed cells x n_steps and the number of blocks
 * (2D: one block = one TB-step launch of the whole grid; 3D: one block = one
 * time step), then forgets the records when reset != 0. At most 4096 runs
 * are recorded between resets. No reference counterpart: it gives
 * benchmarks a per-launch kernel time measured inside their own timed
 * region. */
int gdn_tm_loop_stats(double* loop_ms, double* cell_steps, int64_t* blocks, int32_t reset);

/* ------------------------------------------------------------------------ */
/* 2D TM                                                                    */
/* ------------------------------------------------------------------------ */

/* Scalar description of one 2D TM run. Mirrors the reference SimParams
 * (rust/src/lib.rs:56-69, native.py:124-137) plus the scalars the Rust entry
 * point took by value (lib.rs:123-129). */
typedef struct GdnTmParams {
  int32_t nx, ny;          /* Ez grid, >= 3 each and > 2*npml + 2            */
  int32_t npml;            /* CPML thickness (cells per side), 0 = PEC box    */
  int32_t n_steps;         /* time steps                                      */
  int32_t n_sources;       /* Jz line sources (Ez cells)                      */
  int32_t n_ports;         /* lumped RVS ports (Ez cells)                     */
  int32_t n_mx, n_my;      /* magnetic-current sources on the Hx / Hy grids   */
  int32_t n_probes;        /* Ez probes                                       */
  int32_t n_freq;          /* running-DFT frequencies (0 = no DFT)            */
  int32_t record_energy;   /* 1: write the total field energy every step      */
  int32_t dft_f64;         /* 1: complex128 accumulators, 0: complex64        */
  int32_t cw_sources;      /* 1: Jz/Mx/My waveforms synthesised on the device
                              from per-source CW phasor weights (see buffers) */
  int32_t n_monitors;      /* 0: full-grid DFT into dft_ez/hx/hy; >0: only the
                              boxes listed in GdnTmPoints.monitors             */
  double dt, dx, dy, dz;   /* dz = unit length of the 2D slice (DZ = 1 m)     */
  double mu0;              /* vacuum permeability used by the energy record   */
} GdnTmParams;

/* A running-DFT monitor: the box [lo, hi) of one field component, in that
 * component's own index space (2D uses the first two axes). `out` is a
 * DEVICE buffer of n_freq x box-shape complex values (complex64 or
 * complex128 per dft_f64), written already scaled by dt. Region-limited
 * monitors are the 2D/3D analogue of the reference's DFTRegions
 * (src/gradenna/dft_region.py:37-92). */
typedef struct GdnDftMonitor {
  int32_t comp;            /* 2D: 0 ez, 1 hx, 2 hy; 3D: 0..5 = ex ey ez hx hy hz */
  int32_t lo[3], hi[3];
  void* out;
} GdnDftMonitor;

/* Host-memory point lists (int32 pairs split into i and j arrays). */
typedef struct GdnTmPoints {
  const int32_t *src_i, *src_j;     /* n_sources, margin 1                    */
  const int32_t *port_i, *port_j;   /* n_ports, margin 1                      */
  const int32_t *mx_i, *mx_j;       /* n_mx, on the Hx grid (nx, ny-1)        */
  const int32_t *my_i, *my_j;       /* n_my, on the Hy grid (nx-1, ny)        */
  const int32_t *probe_i, *probe_j; /* n_probes, margin 0                     */
  const GdnDftMonitor* monitors;    /* n_monitors (host array)                */
} GdnTmPoints;

/* Device buffers. Field-typed arrays are float for *_f32, double for *_f64.
 * Argument-for-argument this is the reference's pointer list
 * (native.py:152-170 / lib.rs:96-142), grouped. */
typedef struct GdnTmBuffers {
  const void *ca, *cb, *eps;               /* (nx, ny); eps only if energy    */
  const void *inv_kx_e, *inv_ky_e;         /* (nx-2), (ny-2)                  */
  const void *inv_kx_h, *inv_ky_h;         /* (nx-1), (ny-1)                  */
  /* CPML slab b/c tables, each of length npml: ezx, ezy, hyx, hxy x lo/hi */
  const void *b_ezx_lo, *c_ezx_lo, *b_ezx_hi, *c_ezx_hi;
  const void *b_ezy_lo, *c_ezy_lo, *b_ezy_hi, *c_ezy_hi;
  const void *b_hyx_lo, *c_hyx_lo, *b_hyx_hi, *c_hyx_hi;
  const void *b_hxy_lo, *c_hxy_lo, *b_hxy_hi, *c_hxy_hi;
  double dt_mu, inv_dx, inv_dy;            /* scalars, cast to the field type */
  const void *cb_src;                      /* (n_sources)                     */
  const void *src_cur;                     /* (n_steps, n_sources)            */
  const void *cb_vs;                       /* (n_ports)                       */
  const void *port_vs;                     /* (n_steps, n_ports)              */
  const void *mx_cur, *my_cur;             /* (n_steps, n_mx), (n_steps, n_my)*/
  /* CW-source mode (cw_sources = 1): waveforms are
   *   J_m(n) = env[n] * sum_k Re(W[m,k] * exp(+i w_k t_n))
   * with t_n = (n+1) dt for Jz and (n+1/2) dt for Mx/My; W is complex128
   * (n_src, n_freq); exp(+i w t) is the conjugate of ph_e / ph_h. In this
   * mode src_cur / mx_cur / my_cur are ignored. */
  const double *cw_env;                    /* (n_steps)                       */
  const double *src_w, *mx_w, *my_w;       /* complex128 (n, n_freq)          */
  /* Exact-phase tables exp(-2 pi i f t_n), complex128 (n_steps, n_freq):
   * t_n = (n+1) dt for ph_e, (n+1/2) dt for ph_h (fdtd2d.py:393-398). */
  const double *ph_e, *ph_h;
  /* outputs */
  void *ez, *hx, *hy;                      /* final fields                    */
  void *out_probe;                         /* (n_steps, n_probes)             */
  void *out_v, *out_i;                     /* (n_steps, n_ports)              */
  void *out_energy;                        /* (n_steps)                       */
  void *dft_ez, *dft_hx, *dft_hy;          /* (n_freq, region shape), x dt    */
  void *workspace;                         /* NULL: allocated by the library  */
  size_t workspace_bytes;
} GdnTmBuffers;

/* Scratch bytes needed by gdn_tm_run_* for these parameters and points (the
 * monitor list sizes the DFT monitor ring; pts may be NULL without
 * monitors). */
int gdn_tm_workspace_size(const GdnTmParams* p, const GdnTmPoints* pts, int f64, size_t* bytes);

/* Run the whole 2D TM time loop (replaces gradenna_tm_run_f32/_f64,
 * rust/src/lib.rs:89-641). Stream-ordered; host index lists are consumed
 * before return. */
int gdn_tm_run_f32(const GdnTmParams* p, const GdnTmPoints* pts,
                   const GdnTmBuffers* b, void* stream);
int gdn_tm_run_f64(const GdnTmParams* p, const GdnTmPoints* pts,
                   const GdnTmBuffers* b, void* stream);

/* One problem of a batched run: the same three structs as gdn_tm_run_f32. */
typedef struct GdnTmProblem {
  const GdnTmParams* params;
  const GdnTmPoints* points;
  const GdnTmBuffers* buffers;
} GdnTmProblem;

/* Number of tile configurations a batched run can be forced to (cfg in
 * [0, GDN_TM_NCFG)): 0 = 64x64 tiles, 4-step blocks; 1 = 32x64, 4;
 * 2 = 16x32, 4; 3 = 64x64, 2; 4 = 32x64, 2 (float32 tile sizes). */
#define GDN_TM_NCFG 5

/* Run n independent float32 2D problems together (no reference counterpart:
 * the reference runs one simulation per call). Every problem keeps its own
 * grid, CPML, sources, ports, monitors and n_steps; each block of time
 * steps is ONE launch per tile class over the tiles of all problems still
 * running, so a population of small uneven grids fills the GPU. Results are
 * identical to n separate gdn_tm_run_f32 calls with the same tile
 * configuration. cfg = -1 picks the heuristic configuration of the largest
 * problem; an autotuner passes the fastest measured one. Workspaces: a
 * problem's buffers->workspace if given (gdn_tm_workspace_size bytes), else
 * a stream-ordered block allocated for the call. record_energy is not
 * supported in batched runs (GDN_ERR_BAD_ARG). */
int gdn_tm_run_batch_f32(const GdnTmProblem* problems, int32_t n, int32_t cfg, void* stream);

/* Allocation-free variant of gdn_tm_run_f32. No counterpart in the
 * reference: it exists for callers that must not allocate device memory
 * while they run the solver -- code that owns all GPU memory through its own
 * pool, real-time loops that forbid allocator calls, and hosts that load
 * this library without a CUDA allocator they may use. The caller still
 * passes every input and output buffer; the scratch (field ring, psi slabs,
 * point bins, step counter) lives in a fixed 32 MiB __device__ array inside
 * the library, which every GPU that loads the library holds until the
 * process exits. b->workspace is ignored and nothing is allocated: no
 * cudaMalloc/cudaFree, no graph instantiation (kernels are launched directly
 * on `stream`).
 *   - Runs whose scratch exceeds 32 MiB are rejected with GDN_ERR_BAD_ARG and
 *     a message giving the bytes needed. With the default kernel settings
 *     that is square grids up to about 670 x 670 cells without a DFT and
 *     about 500 x 500 with a full-grid DFT (the DFT fold length shrinks to
 *     fit; DFT monitor boxes cost ring space only for their own cells).
 *   - Every call looks up the array's device address with
 *     cudaGetSymbolAddress on the current device. The first call on a device
 *     (or the first use of the library there, under CUDA's lazy module
 *     loading) loads the library's module, which reserves the 32 MiB array
 *     and the module's code on that device: make one warm-up call, before
 *     any stream capture and before handing the rest of the GPU's memory to
 *     a pool. After that a call allocates nothing.
 *   - All calls share the one array and it keeps the last call's contents;
 *     each call clears the state that must start at zero. Calls that overlap
 *     on the GPU (different streams, or other host threads) race on it and
 *     corrupt each other: serialise them. */
int gdn_tm_run_noalloc_f32(const GdnTmParams* p, const GdnTmPoints* pts,
                           const GdnTmBuffers* b, void* stream);

/* ------------------------------------------------------------------------ */
/* 3D Yee                                                                   */
/* ------------------------------------------------------------------------ */

/* One 3D run (replaces SimParams3D, rust/src/lib3d.rs:40-56). Field shapes
 * (src/gradenna/fdtd3d.py:1-13): Ex (nx-1,ny,nz), Ey (nx,ny-1,nz),
 * Ez (nx,ny,nz-1), Hx (nx,ny-1,nz-1), Hy (nx-1,ny,nz-1), Hz (nx-1,ny-1,nz). */
typedef struct GdnYeeParams {
  int32_t nx, ny, nz;      /* cells per axis, >= 3 and > 2*npml + 2          */
  int32_t npml, n_steps;
  int32_t n_src, n_jx, n_jy;      /* Jz (Ez edges), Jx (Ex), Jy (Ey) sources  */
  int32_t n_mx, n_my, n_mz;       /* magnetic currents on Hx, Hy, Hz          */
  int32_t n_probes;               /* E probes (Ez unless probe_comp is given)  */
  int32_t has_port;               /* 1: one z-directed RVS port               */
  int32_t n_freq, dft_f64, n_monitors;
  int32_t record_energy, cw_sources;
  double dt, dx, dy, dz, mu0;
} GdnYeeParams;

/* Host-memory index lists: (n, 3) int32 row-major (i, j, k) in each source's
 * own component grid; monitors as for 2D with comp 0..5 = ex ey ez hx hy hz.
 * probe_comp (n_probes values, 0 = Ex, 1 = Ey, 2 = Ez; NULL = every probe on
 * Ez, the reference's probe_ijk) picks the E component each probe records
 * after the E half step; a probe lies on its own component's grid. */
typedef struct GdnYeePoints {
  const int32_t *src, *jx, *jy, *mx, *my, *mz, *probe;
  int32_t port[3];
  const GdnDftMonitor* monitors;
  const int32_t* probe_comp;
} GdnYeePoints;

/* Device buffers (field dtype float for *_f32, double for *_f64). The CPML
 * tables are per axis a = x, y, z: E-type (sampled on the PEC interior,
 * n_a - 2 entries) and H-type (half grid, n_a - 1 entries) 1/kappa tables and
 * the slab b/c tables (npml entries, lo/hi), as built by axis_coefficients
 * (src/gradenna/cpml.py:161-208) and sliced by fdtd3d.py:478-503. */
typedef struct GdnYeeBuffers {
  const void *ca, *cb, *eps;              /* (nx, ny, nz) node values          */
  const void *ik_e[3], *ik_h[3];
  const void *b_e_lo[3], *c_e_lo[3], *b_e_hi[3], *c_e_hi[3];
  const void *b_h_lo[3], *c_h_lo[3], *b_h_hi[3], *c_h_hi[3];
  double dt_mu, inv_dx, inv_dy, inv_dz;
  double a_port, b_port, c_port;          /* semi-implicit RVS (fdtd3d.py:517-525) */
  const void *cb_src, *cb_jx, *cb_jy;     /* per source                        */
  const void *src_cur, *jx_cur, *jy_cur;  /* (n_steps, n)                      */
  const void *mx_cur, *my_cur, *mz_cur;   /* (n_steps, n)                      */
  const void *port_vs;                    /* (n_steps)                         */
  const double *cw_env;                   /* CW mode as for 2D (complex128 W)  */
  const double *src_w, *jx_w, *jy_w, *mx_w, *my_w, *mz_w;
  const double *ph_e, *ph_h;              /* complex128 (n_steps, n_freq)      */
  void *ex, *ey, *ez, *hx, *hy, *hz;      /* final fields                      */
  void *out_probe, *out_v, *out_i, *out_energy;
  void *dft[6];                           /* full-grid DFT when n_monitors = 0 */
  void *workspace;
  size_t workspace_bytes;
  /* Resumable runs (NULL = start from rest / keep nothing): the complete
   * time-stepping state, the six fields and the twelve CPML psi arrays, as an
   * opaque DEVICE blob of gdn_yee_state_size bytes. state_in is the state
   * the run starts from (the final state of an earlier run on the same grid,
   * CPML and dtype); state_out receives the state after the last step. Every
   * per-step input (currents, port_vs, cw_env, ph_e, ph_h) is indexed by the
   * run's own step counter, so a run resumed at absolute step s takes the
   * rows s, s+1, ... of the whole run's tables, and its DFT outputs are the
   * partial sums over its own steps. */
  const void* state_in;
  void* state_out;
} GdnYeeBuffers;

int gdn_yee_workspace_size(const GdnYeeParams* p, const GdnYeePoints* pts, int f64, size_t* bytes);

/* Bytes of the resumable state blob of a grid (see GdnYeeBuffers.state_in). */
int gdn_yee_state_size(const GdnYeeParams* p, int f64, size_t* bytes);

/* Run the whole 3D time loop (replaces gradenna_3d_run_f32/_f64,
 * rust/src/lib3d.rs:191-828; step semantics of fdtd3d.py:559-679). */
int gdn_yee_run_f32(const GdnYeeParams* p, const GdnYeePoints* pts, const GdnYeeBuffers* b,
                    void* stream);
int gdn_yee_run_f64(const GdnYeeParams* p, const GdnYeePoints* pts, const GdnYeeBuffers* b,
                    void* stream);

/* ------------------------------------------------------------------------ */
/* Objective reductions and the frequency-domain adjoint contraction (2D)   */
/* ------------------------------------------------------------------------ */

/* Outward spectral Poynting flux through the dual-grid rectangle
 * box = (il, ir, jb, jt) (replaces poynting_flux_box_2d,
 * src/gradenna/monitors.py:20-70). dft_* are DEVICE complex phasors of the
 * full-grid shapes (n_freq, nx, ny) / (n_freq, nx, ny-1) / (n_freq, nx-1, ny),
 * complex128 when c128 = 1 else complex64; `out` is DEVICE double (n_freq). */
int gdn_poynting_box_2d(int32_t nx, int32_t ny, int32_t n_freq, const int32_t box[4],
                        double dx, double dy, int32_t c128, const void* dft_ez,
                        const void* dft_hx, const void* dft_hy, double* out, void* stream);

/* Cotangent of gdn_poynting_box_2d: ADDS g_out[k] * dP_k/dconj-phasor
 * (torch's convention, dL/dRe + i dL/dIm) into g_ez / g_hx / g_hy, which have
 * the shapes and complex type of the phasors. g_out is DEVICE double
 * (n_freq). Deterministic (faces are processed in a fixed order). */
int gdn_poynting_box_2d_grad(int32_t nx, int32_t ny, int32_t n_freq, const int32_t box[4],
                             double dx, double dy, int32_t c128, const void* dft_ez,
                             const void* dft_hx, const void* dft_hy, const double* g_out,
                             void* g_ez, void* g_hx, void* g_hy, void* stream);

/* The built-in 2D objective L = w_prad sum_k P_k + w_s11 sum_k |S11_k|^2,
 * P_k the Poynting flux through the dual-grid contour `box` (as
 * gdn_poynting_box_2d) and S11_k = (V - R I)/(V + R I) of the port at Ez cell
 * `port`, with V and I rebuilt from the field phasors (freq_adjoint.py:536-558;
 * monitors.py:20-70; sparams.py:68-79). It reads the forward run's DFT
 * monitor outputs directly (complex128; any monitor set that covers the
 * contour's Ez strips, Hx/Hy lines and the port's Ez, Hx, Hy cells) and, in
 * one launch, writes the value, P_k, S11_k and the adjoint run's CW source
 * weights: W = conj(dL/dphasor) times the Jz basis -1/cb0 (cb0 = (dt/eps0)/
 * (dx dy)) on the Ez cells and the magnetic basis Q_MAG/(-dt/mu0) on the Hx
 * and Hy cells (freq_adjoint.py:317-352), one row of n_freq complex128 per
 * cell of the lists gdn_tm_objective_cells returns. This replaces scattering
 * the phasors onto full grids and differentiating the objective with torch. */
typedef struct GdnTmObjective {
  int32_t n_freq;
  int32_t box[4];                    /* il, ir, jb, jt                          */
  int32_t port[2];                   /* Ez cell (i, j) of the S11 port          */
  int32_t nx, ny;
  int32_t n_monitors;
  const GdnDftMonitor* monitors;     /* host list; out = DEVICE complex128     */
  const double* freqs;               /* host, n_freq                            */
  double dx, dy, dt, dz, resistance, w_prad, w_s11, eps0, mu0;
  double* value;                     /* DEVICE, 1                               */
  double* p_rad;                     /* DEVICE, n_freq (may be NULL)            */
  void* s11;                         /* DEVICE complex128 n_freq (may be NULL)  */
  void *w_ez, *w_hx, *w_hy;          /* DEVICE complex128 (cells, n_freq)       */
} GdnTmObjective;

/* The objective's cell lists (host int32 (i, j) pairs), in the row order of
 * w_ez / w_hx / w_hy. Call with NULL lists to get the counts. */
int gdn_tm_objective_cells(const GdnTmObjective* o, int32_t* n_ez, int32_t* n_hx, int32_t* n_hy,
                           int32_t* ez_ij, int32_t* hx_ij, int32_t* hy_ij);
int gdn_tm_objective_prad_s11(const GdnTmObjective* o, void* stream);

/* Design-cell gradient of the frequency-domain adjoint (replaces the numpy
 * contraction of freq_adjoint_gradient, src/gradenna/freq_adjoint.py:454-493):
 *   dL/dtheta = s * sum_k k_norm Re[conj(lam_k) conj(G_k)],
 *   G_k = dca E_k / z_k + dcb (E_k - ca E_k / z_k) / cb,  z_k = exp(i w_k dt),
 * with the closed-form dca, dcb of freq_adjoint.py:186-206 and s = eps_r (the
 * reference's scaling, exact only for h = sigma dt / (2 eps) << 1) or, with
 * GDN_CONTRACT_EXACT_LOSS in flags, s = eps_r (1 + h) (exact for any sigma).
 * All arrays are DEVICE: e_fwd, lam (n_freq, n_cells) complex128; eps_r,
 * sigma (n_cells) double; z (n_freq) complex128; grad_sigma / grad_eps_r
 * (n_cells) double, either may be NULL. */
#define GDN_CONTRACT_EXACT_LOSS 1
int gdn_tm_adjoint_contract(int32_t n_cells, int32_t n_freq, double dt, double k_norm,
                            const void* e_fwd, const void* lam, const double* eps_r,
                            const double* sigma, const void* z, double* grad_sigma,
                            double* grad_eps_r, int32_t flags, void* stream);

/* ------------------------------------------------------------------------ */
/* Near-to-far-field projection (3D and 2D)                                 */
/* ------------------------------------------------------------------------ */

/* Radiation vectors and far-field pattern amplitudes of equivalent surface
 * currents (replaces the einsum core of ntff_3d, src/gradenna/ntff.py:399-428):
 *   N_d = sum_p w_p exp(+i k rhat_d . r_p) J_p,  L_d likewise with M_p,
 *   E_theta = -(i k / 4 pi)(L_phi + eta0 N_theta),
 *   E_phi   = +(i k / 4 pi)(L_theta - eta0 N_phi).
 * DEVICE arrays, complex128 when c128 = 1 else complex64 for J, M, out:
 *   pos (n_pts, 3) double, w (n_pts) double, J/M (n_freq, n_pts, 3),
 *   k (n_freq) double, dirs (n_dir, 4) double = (cos th, sin th, cos ph, sin ph),
 *   out (n_freq, n_dir, 2) = (E_theta, E_phi). */
int gdn_ntff3d_project(int32_t n_freq, int32_t n_pts, int32_t n_dir, int32_t c128,
                       const double* pos, const double* w, const void* J, const void* M,
                       const double* k, const double* dirs, double eta0, void* out,
                       void* stream);

/* Adjoint of gdn_ntff3d_project: given g_out (n_freq, n_dir, 2) in torch's
 * complex-gradient convention, WRITES g_J, g_M (n_freq, n_pts, 3). */
int gdn_ntff3d_project_grad(int32_t n_freq, int32_t n_pts, int32_t n_dir, int32_t c128,
                            const double* pos, const double* w, const double* k,
                            const double* dirs, double eta0, const void* g_out, void* g_J,
                            void* g_M, void* stream);

/* 2D contour projection (ntff_2d, src/gradenna/ntff.py:213-228):
 *   E_far(f, phi) = pref_f sum_p w_p (eta0 Jz_p - (n_p . u_phi) Ez_p)
 *                   exp(+i k (x_p cos phi + y_p sin phi)),
 * pref_f = -sqrt(i k / 8 pi). pos (n_pts, 4) double = (x, y, n_x, n_y);
 * Jz, Ez (n_freq, n_pts); angles (n_ang) double; out (n_freq, n_ang). */
int gdn_ntff2d_project(int32_t n_freq, int32_t n_pts, int32_t n_ang, int32_t c128,
                       const double* pos, const double* w, const void* Jz, const void* Ez,
                       const double* k, const double* angles, double eta0, void* out,
                       void* stream);

/* Adjoint of gdn_ntff2d_project: given g_out (n_freq, n_ang) in torch's
 * complex-gradient convention, WRITES g_Jz, g_Ez (n_freq, n_pts). */
int gdn_ntff2d_project_grad(int32_t n_freq, int32_t n_pts, int32_t n_ang, int32_t c128,
                            const double* pos, const double* w, const double* k,
                            const double* angles, double eta0, const void* g_out, void* g_Jz,
                            void* g_Ez, void* stream);

/* ---- Design surrogate (BF16 U-Net) kernels ----------------------------
 * No reference counterpart (the reference has no learned component).
 * Activations are NHWC bfloat16; a tensor may be the channel slice
 * [c0, c0 + C) of a buffer whose rows hold `stride` channels. Weights are
 * bfloat16 [taps * Cin][Cout], row k = tap * Cin + ci with
 * tap = (dy + 1) * 3 + (dx + 1) (taps = 9) or 0 (taps = 1); zero padding. */

/* out = act(bias + conv(in, w)): bf16 `out` (slice) and/or float32 `out32`
 * (dense [P][Cout]); bias float32 or NULL; relu 0/1 selects the leaky ReLU
 * act(x) = x > 0 ? x : slope x (slope 0 = ReLU). With `mask` non-NULL,
 * outputs whose mask entry is <= 0 are multiplied by slope (the activation
 * derivative when this is an input-gradient convolution). */
int gdn_sur_conv_fwd(const void* in, int32_t in_stride, int32_t in_c0, int32_t N, int32_t H,
                     int32_t W, int32_t Cin, int32_t taps, const void* w, const float* bias,
                     int32_t Cout, int32_t relu, float slope, void* out, int32_t out_stride,
                     int32_t out_c0,
                     float* out32, const void* mask, int32_t mask_stride, int32_t mask_c0,
                     void* stream);

/* dw[k][co] += sum_p im2col(in)[p][k] g[p][co] and db[co] += sum_p g[p][co]
 * (float32, accumulated; db may be NULL). */
int gdn_sur_conv_wgrad(const void* in, int32_t in_stride, int32_t in_c0, int32_t N, int32_t H,
                       int32_t W, int32_t Cin, int32_t taps, const void* g, int32_t g_stride,
                       int32_t g_c0, int32_t Cout, float* dw, float* db, void* stream);

/* Weights of the input-gradient convolution (Cin and Cout swapped, taps
 * point-reflected): wt[(taps-1-tap) * Cout + co][ci] = w[tap * Cin + ci][co]. */
int gdn_sur_flip_weights(const void* w, int32_t Cin, int32_t Cout, int32_t taps, void* wt,
                         void* stream);

/* 2x2 max pooling (H, W even) with the winning window position (uint8). */
int gdn_sur_maxpool2(const void* in, int32_t in_stride, int32_t in_c0, int32_t N, int32_t H,
                     int32_t W, int32_t C, void* out, void* arg, void* stream);

/* gin[winner] += gout for the pooling of an (N, H, W, C) slice. */
int gdn_sur_maxpool2_grad_acc(const void* gout, const void* arg, int32_t N, int32_t H,
                              int32_t W, int32_t C, void* gin, int32_t gin_stride,
                              int32_t gin_c0, void* stream);

/* Nearest x2 upsampling of a dense (N, H, W, C) tensor into a slice, and the
 * gradient (sum of the four copies) back to a dense (N, H, W, C) tensor. */
int gdn_sur_upsample2(const void* in, int32_t N, int32_t H, int32_t W, int32_t C, void* out,
                      int32_t out_stride, int32_t out_c0, void* stream);
int gdn_sur_upsample2_grad(const void* gout, int32_t g_stride, int32_t g_c0, int32_t N,
                           int32_t H, int32_t W, int32_t C, void* gin, void* stream);

/* Head loss gradient for out32 (N, HW, C >= 3): channels 0, 1 = field,
 * channel 2 = power density (predicted power = its mean over HW, written to
 * mean[N]). With targets, L = wf mean (out[:2] - target_field)^2 +
 * wp mean_n (mean_n - target_power_n)^2 is added to *loss (may be NULL);
 * without (both NULL), grad = d(sum_n power_weight_n mean_n)/d out
 * (power_weight NULL = 1). Writes the bf16 gradient (N, HW, C). */
int gdn_sur_head_grad(const float* out32, int32_t N, int32_t HW, int32_t C,
                      const float* target_field, const float* target_power,
                      const float* power_weight, float wf, float wp, float* mean, void* grad,
                      float* loss, void* stream);

/* One Adam step on float32 master weights w (n) with gradient g and moments
 * m, v, refreshing the bf16 copy w16 (may be NULL). hyper (device float[4])
 * = {step, lr, 1 - b1^step, 1 - b2^step}: the step count is advanced on the
 * device, so the call can be captured in a CUDA graph. */
int gdn_sur_adam(float* w, const float* g, float* m, float* v, void* w16, int64_t n,
                 float* hyper, float b1, float b2, float eps, void* stream);

/* float32 -> bfloat16 conversion of n elements. */
int gdn_sur_to_bf16(const float* a, void* b, int64_t n, void* stream);

/* gdn_sur_conv_fwd on the tcgen05 tensor cores (TMEM accumulators, 128-pixel
 * tiles, 128-byte-swizzled K-major operands staged by cp.async). Same
 * arguments and results, except the weights `wk` are K-major: [Cout][K]
 * (see gdn_sur_weights_kmajor). Needs Cin, in_stride and in_c0 multiples of
 * 8 and 16-byte aligned `in` and `wk`. Its mbarrier waits are bounded; a
 * wait that runs out is recorded for gdn_sur_status. */
int gdn_sur_conv_fwd_tc(const void* in, int32_t in_stride, int32_t in_c0, int32_t N, int32_t H,
                        int32_t W, int32_t Cin, int32_t taps, const void* wk, const float* bias,
                        int32_t Cout, int32_t relu, float slope, void* out, int32_t out_stride,
                        int32_t out_c0, float* out32, const void* mask, int32_t mask_stride,
                        int32_t mask_c0, void* stream);

/* K-major weights for gdn_sur_conv_fwd_tc from [taps * Cin][Cout] weights w:
 * flip = 0: the layer's own convolution, wk[co][tap * Cin + ci];
 * flip = 1: its input-gradient convolution (Cin and Cout swapped, taps
 * point-reflected), wk[ci][(taps - 1 - tap) * Cout + co]. */
int gdn_sur_weights_kmajor(const void* w, int32_t Cin, int32_t Cout, int32_t taps, int32_t flip,
                           void* wk, void* stream);

/* ---- Topology-optimisation design transform ----------------------------
 * rho = tanh_projection(conic_filter(sigmoid(theta), R), beta, eta) for B
 * designs of H x W cells (src/gradenna/topopt.py:55-127, which runs in jax).
 * kern: the (2n+1)^2 conic weights max(0, 1 - |o| / R), n <= 24; the
 * filter is renormalised by the in-bounds weight sum at the border. All
 * arrays are DEVICE double, (B, H, W). The forward also writes the filtered
 * field and the per-cell weight sum, which the backward reads to turn
 * g_rho = dL/drho into g_theta = dL/dtheta. */
int gdn_design_forward(const double* theta, int32_t B, int32_t H, int32_t W, const double* kern,
                       int32_t n, double beta, double eta, double* filt, double* norm,
                       double* rho, void* stream);
int gdn_design_backward(const double* theta, const double* filt, const double* norm,
                        const double* g_rho, int32_t B, int32_t H, int32_t W, const double* kern,
                        int32_t n, double beta, double eta, double* g_theta, void* stream);

/* Number of tensor-core convolutions whose bounded waits ran out since the
 * last reset (0 in normal operation); synchronises with the device. */
int gdn_sur_status(int32_t* timeouts, int32_t reset);

/* Test hook for the abort path of gdn_sur_conv_fwd_tc. With step >= 0 every
 * CTA of the following tensor-core convolutions gives up at that reduction
 * step as if a stage wait had run out: it waits (bounded) for the MMAs it
 * already issued, releases its TMEM, writes no results and is counted by
 * gdn_sur_status. step = -1 (the default) switches the hook off. */
int gdn_sur_inject_timeout(int32_t step);

#ifdef __cplusplus
}
#endif

#endif /* GRADENNA_B200_H */
