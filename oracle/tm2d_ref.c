/* C restatement of the reference 2D TM time loop (test oracle and CPU
 * baseline only; never part of the product).
 *
 * Exports oracle_tm_run_f32 / oracle_tm_run_f64 taking the same structs as
 * the CUDA entry points (include/gradenna_b200.h) but with HOST pointers,
 * so tests and bench.py can drive both with one set of buffers. Threads:
 * OpenMP (OMP_NUM_THREADS). */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/gradenna_b200.h"

/* Source waveform at step n: tabulated, or CW-synthesised
 * J(n) = env[n] Re(sum_k W_k conj(ph[n,k])) (freq_adjoint.py:317-352). */
#define REAL float
#define FN(x) x##_f32
static REAL FN(wave)(const GdnTmParams* p, const GdnTmBuffers* b, const REAL* cur, const double* w,
                     const double* ph, int npts, int m, int n) {
  if (!p->cw_sources) return cur[(size_t)n * npts + m];
  double s = 0.0;
  for (int k = 0; k < p->n_freq; ++k)
    s += w[2 * ((size_t)m * p->n_freq + k)] * ph[2 * ((size_t)n * p->n_freq + k)] +
         w[2 * ((size_t)m * p->n_freq + k) + 1] * ph[2 * ((size_t)n * p->n_freq + k) + 1];
  return (REAL)(b->cw_env[n] * s);
}
#include "tm2d_body.h"
#undef REAL
#undef FN

#define REAL double
#define FN(x) x##_f64
static REAL FN(wave)(const GdnTmParams* p, const GdnTmBuffers* b, const REAL* cur, const double* w,
                     const double* ph, int npts, int m, int n) {
  if (!p->cw_sources) return cur[(size_t)n * npts + m];
  double s = 0.0;
  for (int k = 0; k < p->n_freq; ++k)
    s += w[2 * ((size_t)m * p->n_freq + k)] * ph[2 * ((size_t)n * p->n_freq + k)] +
         w[2 * ((size_t)m * p->n_freq + k) + 1] * ph[2 * ((size_t)n * p->n_freq + k) + 1];
  return (REAL)(b->cw_env[n] * s);
}
#include "tm2d_body.h"
#undef REAL
#undef FN

int oracle_tm_run_f32(const GdnTmParams* p, const GdnTmPoints* pt, const GdnTmBuffers* b) {
  return run_f32(p, pt, b);
}
int oracle_tm_run_f64(const GdnTmParams* p, const GdnTmPoints* pt, const GdnTmBuffers* b) {
  return run_f64(p, pt, b);
}
