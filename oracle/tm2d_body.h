/* Body of the C restatement of the reference 2D TM time loop, instantiated
 * for REAL = float and REAL = double by tm2d_ref.c (test/baseline oracle).
 *
 * Step order and arithmetic follow src/gradenna/fdtd2d.py:412-464 (the same
 * order the reference's fused CPU kernel rust/src/lib.rs:293-615 uses):
 * H sweep with slab psi -> Mx/My -> port current + Ez^n -> E sweep with psi
 * -> Jz -> port injection + V -> DFT (double accumulators) -> probes ->
 * energy. Rows are split across OpenMP threads; point work is serial.
 *
 * All pointers in the GdnTm* structs are HOST pointers here. */

static int FN(run)(const GdnTmParams* p, const GdnTmPoints* pt, const GdnTmBuffers* b) {
  const int nx = p->nx, ny = p->ny, npml = p->npml, N = p->n_steps, K = p->n_freq;
  const REAL* ca = (const REAL*)b->ca;
  const REAL* cb = (const REAL*)b->cb;
  const REAL* eps = (const REAL*)b->eps;
  const REAL *ikx_e = (const REAL*)b->inv_kx_e, *iky_e = (const REAL*)b->inv_ky_e;
  const REAL *ikx_h = (const REAL*)b->inv_kx_h, *iky_h = (const REAL*)b->inv_ky_h;
  const REAL *b_ezx_lo = (const REAL*)b->b_ezx_lo, *c_ezx_lo = (const REAL*)b->c_ezx_lo;
  const REAL *b_ezx_hi = (const REAL*)b->b_ezx_hi, *c_ezx_hi = (const REAL*)b->c_ezx_hi;
  const REAL *b_ezy_lo = (const REAL*)b->b_ezy_lo, *c_ezy_lo = (const REAL*)b->c_ezy_lo;
  const REAL *b_ezy_hi = (const REAL*)b->b_ezy_hi, *c_ezy_hi = (const REAL*)b->c_ezy_hi;
  const REAL *b_hyx_lo = (const REAL*)b->b_hyx_lo, *c_hyx_lo = (const REAL*)b->c_hyx_lo;
  const REAL *b_hyx_hi = (const REAL*)b->b_hyx_hi, *c_hyx_hi = (const REAL*)b->c_hyx_hi;
  const REAL *b_hxy_lo = (const REAL*)b->b_hxy_lo, *c_hxy_lo = (const REAL*)b->c_hxy_lo;
  const REAL *b_hxy_hi = (const REAL*)b->b_hxy_hi, *c_hxy_hi = (const REAL*)b->c_hxy_hi;
  const REAL dt_mu = (REAL)b->dt_mu, inv_dx = (REAL)b->inv_dx, inv_dy = (REAL)b->inv_dy;
  const REAL dx = (REAL)p->dx, dy = (REAL)p->dy, dz = (REAL)p->dz;
  const int ns = p->n_sources, np_ = p->n_ports, nmx = p->n_mx, nmy = p->n_my, npr = p->n_probes;
  const REAL *cb_src = (const REAL*)b->cb_src, *src_cur = (const REAL*)b->src_cur;
  const REAL *cb_vs = (const REAL*)b->cb_vs, *port_vs = (const REAL*)b->port_vs;
  const REAL *mx_cur = (const REAL*)b->mx_cur, *my_cur = (const REAL*)b->my_cur;
  const double* ph_e = b->ph_e;
  const double* ph_h = b->ph_h;
  REAL *out_probe = (REAL*)b->out_probe, *out_v = (REAL*)b->out_v, *out_i = (REAL*)b->out_i;
  REAL* out_energy = (REAL*)b->out_energy;

  const size_t ne = (size_t)nx * ny, nhx = (size_t)nx * (ny - 1), nhy = (size_t)(nx - 1) * ny;
  REAL* ez = (REAL*)calloc(ne, sizeof(REAL));
  REAL* hx = (REAL*)calloc(nhx, sizeof(REAL));
  REAL* hy = (REAL*)calloc(nhy, sizeof(REAL));
  const int ni = nx - 2, nj = ny - 2;
  REAL* ezx_lo = (REAL*)calloc((size_t)npml * nj + 1, sizeof(REAL));
  REAL* ezx_hi = (REAL*)calloc((size_t)npml * nj + 1, sizeof(REAL));
  REAL* ezy_lo = (REAL*)calloc((size_t)ni * npml + 1, sizeof(REAL));
  REAL* ezy_hi = (REAL*)calloc((size_t)ni * npml + 1, sizeof(REAL));
  REAL* hyx_lo = (REAL*)calloc((size_t)npml * ny + 1, sizeof(REAL));
  REAL* hyx_hi = (REAL*)calloc((size_t)npml * ny + 1, sizeof(REAL));
  REAL* hxy_lo = (REAL*)calloc((size_t)nx * npml + 1, sizeof(REAL));
  REAL* hxy_hi = (REAL*)calloc((size_t)nx * npml + 1, sizeof(REAL));
  REAL* ez_before = (REAL*)calloc((size_t)np_ + 1, sizeof(REAL));

  /* DFT monitors (double accumulators, interleaved re/im). */
  int nmon = 0;
  int mcomp[64], mlo0[64], mlo1[64], mh[64], mw[64];
  double* macc[64];
  if (K > 0) {
    if (p->n_monitors == 0) {
      const int shp[3][2] = {{nx, ny}, {nx, ny - 1}, {nx - 1, ny}};
      for (int c = 0; c < 3; ++c) {
        mcomp[c] = c; mlo0[c] = 0; mlo1[c] = 0; mh[c] = shp[c][0]; mw[c] = shp[c][1];
      }
      nmon = 3;
    } else {
      nmon = p->n_monitors > 64 ? 64 : p->n_monitors;
      for (int m = 0; m < nmon; ++m) {
        const GdnDftMonitor* mo = &pt->monitors[m];
        mcomp[m] = mo->comp; mlo0[m] = mo->lo[0]; mlo1[m] = mo->lo[1];
        mh[m] = mo->hi[0] - mo->lo[0]; mw[m] = mo->hi[1] - mo->lo[1];
      }
    }
    for (int m = 0; m < nmon; ++m) macc[m] = (double*)calloc((size_t)2 * K * mh[m] * mw[m], sizeof(double));
  }

  for (int n = 0; n < N; ++n) {
    /* (1) H sweep (fdtd2d.py:416-428). */
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i) {
      for (int j = 0; j < ny - 1; ++j) {
        const REAL diff = (ez[(size_t)i * ny + j + 1] - ez[(size_t)i * ny + j]) * inv_dy;
        REAL term = diff;
        if (j < npml) {
          REAL* ps = &hxy_lo[(size_t)i * npml + j];
          *ps = b_hxy_lo[j] * *ps + c_hxy_lo[j] * diff;
          term = diff * iky_h[j] + *ps;
        } else if (j >= ny - 1 - npml) {
          const int s = j - (ny - 1 - npml);
          REAL* ps = &hxy_hi[(size_t)i * npml + s];
          *ps = b_hxy_hi[s] * *ps + c_hxy_hi[s] * diff;
          term = diff * iky_h[j] + *ps;
        }
        hx[(size_t)i * (ny - 1) + j] -= dt_mu * term;
      }
      if (i < nx - 1) {
        for (int j = 0; j < ny; ++j) {
          const REAL diff = (ez[(size_t)(i + 1) * ny + j] - ez[(size_t)i * ny + j]) * inv_dx;
          REAL term = diff;
          if (i < npml) {
            REAL* ps = &hyx_lo[(size_t)i * ny + j];
            *ps = b_hyx_lo[i] * *ps + c_hyx_lo[i] * diff;
            term = diff * ikx_h[i] + *ps;
          } else if (i >= nx - 1 - npml) {
            const int s = i - (nx - 1 - npml);
            REAL* ps = &hyx_hi[(size_t)s * ny + j];
            *ps = b_hyx_hi[s] * *ps + c_hyx_hi[s] * diff;
            term = diff * ikx_h[i] + *ps;
          }
          hy[(size_t)i * ny + j] += dt_mu * term;
        }
      }
    }
    for (int m = 0; m < nmx; ++m)
      hx[(size_t)pt->mx_i[m] * (ny - 1) + pt->mx_j[m]] -= dt_mu * FN(wave)(p, b, mx_cur, b->mx_w, ph_h, nmx, m, n);
    for (int m = 0; m < nmy; ++m)
      hy[(size_t)pt->my_i[m] * ny + pt->my_j[m]] -= dt_mu * FN(wave)(p, b, my_cur, b->my_w, ph_h, nmy, m, n);
    /* (2) port current and Ez^n (fdtd2d.py:430-436). */
    for (int k = 0; k < np_; ++k) {
      const int i = pt->port_i[k], j = pt->port_j[k];
      out_i[(size_t)n * np_ + k] = (hy[(size_t)i * ny + j] - hy[(size_t)(i - 1) * ny + j]) * dy -
                                   (hx[(size_t)i * (ny - 1) + j] - hx[(size_t)i * (ny - 1) + j - 1]) * dx;
      ez_before[k] = ez[(size_t)i * ny + j];
    }
    /* (3) E sweep (fdtd2d.py:438-443). */
#pragma omp parallel for schedule(static)
    for (int a = 0; a < ni; ++a) {
      const int i = a + 1;
      for (int bb = 0; bb < nj; ++bb) {
        const int j = bb + 1;
        const REAL dhy_dx = (hy[(size_t)i * ny + j] - hy[(size_t)(i - 1) * ny + j]) * inv_dx;
        const REAL dhx_dy = (hx[(size_t)i * (ny - 1) + j] - hx[(size_t)i * (ny - 1) + j - 1]) * inv_dy;
        REAL tx = dhy_dx, ty = dhx_dy;
        if (a < npml) {
          REAL* ps = &ezx_lo[(size_t)a * nj + bb];
          *ps = b_ezx_lo[a] * *ps + c_ezx_lo[a] * dhy_dx;
          tx = dhy_dx * ikx_e[a] + *ps;
        } else if (a >= ni - npml) {
          const int s = a - (ni - npml);
          REAL* ps = &ezx_hi[(size_t)s * nj + bb];
          *ps = b_ezx_hi[s] * *ps + c_ezx_hi[s] * dhy_dx;
          tx = dhy_dx * ikx_e[a] + *ps;
        }
        if (bb < npml) {
          REAL* ps = &ezy_lo[(size_t)a * npml + bb];
          *ps = b_ezy_lo[bb] * *ps + c_ezy_lo[bb] * dhx_dy;
          ty = dhx_dy * iky_e[bb] + *ps;
        } else if (bb >= nj - npml) {
          const int s = bb - (nj - npml);
          REAL* ps = &ezy_hi[(size_t)a * npml + s];
          *ps = b_ezy_hi[s] * *ps + c_ezy_hi[s] * dhx_dy;
          ty = dhx_dy * iky_e[bb] + *ps;
        }
        const size_t g = (size_t)i * ny + j;
        ez[g] = ca[g] * ez[g] + cb[g] * (tx - ty);
      }
    }
    /* (4) Jz, ports, V (fdtd2d.py:444-451). */
    for (int m = 0; m < ns; ++m)
      ez[(size_t)pt->src_i[m] * ny + pt->src_j[m]] -= cb_src[m] * FN(wave)(p, b, src_cur, b->src_w, ph_e, ns, m, n);
    for (int k = 0; k < np_; ++k)
      ez[(size_t)pt->port_i[k] * ny + pt->port_j[k]] -= cb_vs[k] * port_vs[(size_t)n * np_ + k];
    for (int k = 0; k < np_; ++k)
      out_v[(size_t)n * np_ + k] = (REAL)(-0.5) * dz * (ez_before[k] + ez[(size_t)pt->port_i[k] * ny + pt->port_j[k]]);
    /* (5) DFT (fdtd2d.py:453-458) with double accumulators. */
    for (int m = 0; m < nmon; ++m) {
      const REAL* f = mcomp[m] == 0 ? ez : (mcomp[m] == 1 ? hx : hy);
      const int fw = mcomp[m] == 1 ? ny - 1 : ny;
      const double* ph = mcomp[m] == 0 ? ph_e : ph_h;
      const int h = mh[m], w = mw[m];
      double* acc = macc[m];
#pragma omp parallel for schedule(static)
      for (int r = 0; r < h; ++r)
        for (int k = 0; k < K; ++k) {
          const double pr = ph[2 * ((size_t)n * K + k)], pi = ph[2 * ((size_t)n * K + k) + 1];
          double* ak = acc + 2 * ((size_t)k * h * w + (size_t)r * w);
          const REAL* fr = f + (size_t)(mlo0[m] + r) * fw + mlo1[m];
          for (int c = 0; c < w; ++c) {
            ak[2 * c] += pr * (double)fr[c];
            ak[2 * c + 1] += pi * (double)fr[c];
          }
        }
    }
    /* (6) probes, energy (fdtd2d.py:160-169, 461-463). */
    for (int k = 0; k < npr; ++k) out_probe[(size_t)n * npr + k] = ez[(size_t)pt->probe_i[k] * ny + pt->probe_j[k]];
    if (p->record_energy) {
      double ue = 0.0, uh = 0.0;
#pragma omp parallel for reduction(+ : ue)
      for (size_t g = 0; g < ne; ++g) ue += (double)eps[g] * (double)ez[g] * (double)ez[g];
#pragma omp parallel for reduction(+ : uh)
      for (size_t g = 0; g < nhx; ++g) uh += (double)hx[g] * (double)hx[g];
#pragma omp parallel for reduction(+ : uh)
      for (size_t g = 0; g < nhy; ++g) uh += (double)hy[g] * (double)hy[g];
      out_energy[n] = (REAL)(0.5 * ue * p->dx * p->dy + 0.5 * p->mu0 * uh * p->dx * p->dy);
    }
  }

  /* Outputs: final fields and dt-scaled DFT (complex64 or complex128). */
  memcpy(b->ez, ez, ne * sizeof(REAL));
  memcpy(b->hx, hx, nhx * sizeof(REAL));
  memcpy(b->hy, hy, nhy * sizeof(REAL));
  for (int m = 0; m < nmon; ++m) {
    void* out = p->n_monitors == 0 ? (mcomp[m] == 0 ? b->dft_ez : (mcomp[m] == 1 ? b->dft_hx : b->dft_hy))
                                   : pt->monitors[m].out;
    const size_t cnt = (size_t)2 * K * mh[m] * mw[m];
    for (size_t q = 0; q < cnt; ++q) {
      if (p->dft_f64)
        ((double*)out)[q] = macc[m][q] * p->dt;
      else
        ((float*)out)[q] = (float)(macc[m][q] * p->dt);
    }
    free(macc[m]);
  }
  free(ez); free(hx); free(hy); free(ez_before);
  free(ezx_lo); free(ezx_hi); free(ezy_lo); free(ezy_hi);
  free(hyx_lo); free(hyx_hi); free(hxy_lo); free(hxy_hi);
  return 0;
}
