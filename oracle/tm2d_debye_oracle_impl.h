/*
 * TEST INFRASTRUCTURE ONLY.  CPU oracle of the Debye-medium TM2D forward with
 * storage and of its exact discrete adjoint (included by tm2d_oracle.c after
 * tm2d_oracle_impl.h, once per REAL).
 *
 * Forward: the reference's Debye time step (maxwell_tm_cuda_inst.cu:382-457
 * and the Python reference tm2d_python.py:481-503): per cell of the update
 * domain, e1 = ca E + cb curlH + sum_p cp_p P_p, sources added, then
 * P_p <- a_p P_p + b_p (e1 + E), E <- e1.
 *
 * Adjoint: the reference has no native Debye adjoint (it differentiates the
 * Python time loop with torch autograd); this is the exact transpose of the
 * step above, written out by hand (see include/tide_b200_debye.h for the
 * recursion), pinned against the reference's autograd gradients by
 * tests/test_debye_oracle.py.  Arguments: the TideTMDebye struct of
 * include/tide_b200_debye.h (host pointers here).
 */

#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

static void FN(debye_geom)(const TideTMDebye *A, FN(geom) * g) {
  const REAL *const *pr = (const REAL *const *)A->profiles;
  g->ay = pr[0]; g->by = pr[1]; g->ayh = pr[2]; g->byh = pr[3];
  g->ax = pr[4]; g->bx = pr[5]; g->axh = pr[6]; g->bxh = pr[7];
  g->ky = pr[8]; g->kyh = pr[9]; g->kx = pr[10]; g->kxh = pr[11];
  g->rdy = (REAL)A->rdy; g->rdx = (REAL)A->rdx;
  g->n_shots = A->n_shots; g->ny = A->ny; g->nx = A->nx;
  g->n_src = A->n_src; g->n_rec = A->n_rec;
  g->pml_y0 = A->pml_y0; g->pml_x0 = A->pml_x0; g->pml_y1 = A->pml_y1; g->pml_x1 = A->pml_x1;
  g->stencil = (int)A->stencil;
  g->ca_b = g->cb_b = g->cq_b = false;
}

static inline void FN(debye_put)(void *store, bool bf16, int64_t idx, REAL v) {
  if (!store) return;
  if (bf16)
    ((uint16_t *)store)[idx] = FN(to_bf16)(v);
  else
    ((REAL *)store)[idx] = v;
}
static inline REAL FN(debye_get)(const void *store, bool bf16, int64_t idx) {
  return bf16 ? FN(from_bf16)(((const uint16_t *)store)[idx]) : ((const REAL *)store)[idx];
}

void FN(tide_oracle_tm_debye_forward_with_storage)(const TideTMDebye *A) {
  FN(geom) g;
  FN(debye_geom)(A, &g);
  const int64_t S = A->n_shots, ny = A->ny, nx = A->nx, N = ny * nx, NP = A->n_poles;
  const int p = (int)A->stencil / 2;
  const bool bf16 = A->storage_format == 1;
  const REAL *ca = A->ca, *cb = A->cb, *cq = A->cq;
  const REAL *da = A->a, *db = A->b, *dcp = A->cp;
  REAL *ey = A->fields[0], *hx = A->fields[1], *hz = A->fields[2];
  REAL *m_ey_x = A->fields[3], *m_ey_z = A->fields[4];
  REAL *m_hx_z = A->fields[5], *m_hz_x = A->fields[6];
  REAL *pol = A->pol;
  const int64_t k = A->step_ratio;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < S; ++s) {
    REAL *eprev = (REAL *)malloc((size_t)N * sizeof(REAL));
    for (int64_t t = A->start_t; t < A->start_t + A->nt; ++t) {
      FN(step_h)(&g, cq, ey, hx, hz, m_ey_x, m_ey_z, s);
      const bool store = (t % k) == 0;
      const int64_t q = t / k - A->q0;
      for (int64_t y = p; y < ny - p + 1; ++y) {
        for (int64_t x = p; x < nx - p + 1; ++x) {
          const int64_t j = y * nx + x, i = s * N + j;
          REAL dz = FN(d_x1)(hz, i, g.stencil, g.rdx);
          REAL dy = FN(d_y1)(hx, i, nx, g.stencil, g.rdy);
          if (x < g.pml_x0 || x >= g.pml_x1) {
            m_hz_x[i] = g.bx[x] * m_hz_x[i] + g.ax[x] * dz;
            dz = dz / g.kx[x] + m_hz_x[i];
          }
          if (y < g.pml_y0 || y >= g.pml_y1) {
            m_hx_z[i] = g.by[y] * m_hx_z[i] + g.ay[y] * dy;
            dy = dy / g.ky[y] + m_hx_z[i];
          }
          const REAL curl = dz - dy;
          const REAL eo = ey[i];
          eprev[j] = eo;
          if (store) {
            FN(debye_put)(A->ey_store, bf16, q * S * N + i, eo);
            FN(debye_put)(A->curl_store, bf16, q * S * N + i, curl);
            for (int64_t pp = 0; pp < NP; ++pp)
              FN(debye_put)(A->pol_store, bf16, ((q * S + s) * NP + pp) * N + j,
                            pol[(s * NP + pp) * N + j]);
          }
          REAL e = ca[j] * eo + cb[j] * curl;
          REAL pt = (REAL)0;
          for (int64_t pp = 0; pp < NP; ++pp)
            pt = pt + dcp[pp * N + j] * pol[(s * NP + pp) * N + j];
          ey[i] = e + pt;
        }
      }
      if (A->n_src > 0)
        FN(inject)(ey, (const REAL *)A->f + t * S * A->n_src, A->sources_i, A->n_src, N, s);
      for (int64_t y = p; y < ny - p + 1; ++y) {
        for (int64_t x = p; x < nx - p + 1; ++x) {
          const int64_t j = y * nx + x, i = s * N + j;
          const REAL es = ey[i] + eprev[j];
          if (store) FN(debye_put)(A->esum_store, bf16, q * S * N + i, es);
          for (int64_t pp = 0; pp < NP; ++pp) {
            const int64_t c = pp * N + j, pi = (s * NP + pp) * N + j;
            pol[pi] = da[c] * pol[pi] + db[c] * es;
          }
        }
      }
      if (A->n_rec > 0)
        FN(record)((REAL *)A->r + t * S * A->n_rec, ey, A->receivers_i, A->n_rec, N, s);
    }
    free(eprev);
  }
}

void FN(tide_oracle_tm_debye_backward)(const TideTMDebye *A) {
  FN(geom) g;
  FN(debye_geom)(A, &g);
  const int64_t S = A->n_shots, ny = A->ny, nx = A->nx, N = ny * nx, SN = S * N;
  const int64_t NP = A->n_poles;
  const int p = (int)A->stencil / 2;
  const bool bf16 = A->storage_format == 1;
  const REAL *ca = A->ca, *cb = A->cb, *cq = A->cq;
  const REAL *da = A->a, *db = A->b, *dcp = A->cp;
  REAL *lam_ey = A->lam[0], *lam_hx = A->lam[1], *lam_hz = A->lam[2];
  REAL *lpol = A->lam_pol;
  REAL *scratch = A->scratch;
  memset(scratch, 0, (size_t)4 * SN * sizeof(REAL));
  REAL *U = (REAL *)malloc((size_t)SN * sizeof(REAL));
  REAL *cur_ey_x = A->lam[3], *cur_ey_z = A->lam[4];
  REAL *cur_hx_z = A->lam[5], *cur_hz_x = A->lam[6];
  REAL *nxt_ey_x = scratch, *nxt_ey_z = scratch + SN;
  REAL *nxt_hx_z = scratch + 2 * SN, *nxt_hz_x = scratch + 3 * SN;
  const int64_t k = A->step_ratio;
  const REAL kscale = (REAL)k;
  int64_t swaps = 0;
  for (int64_t t = A->start_t - 1; t >= A->start_t - A->nt; --t) {
    REAL *tmp;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < S; ++s)
      FN(adj_e)(&g, cb, lam_ey, lam_hx, lam_hz, cur_hx_z, cur_hz_x, nxt_hx_z, nxt_hz_x, s);
    tmp = cur_hx_z; cur_hx_z = nxt_hx_z; nxt_hx_z = tmp;
    tmp = cur_hz_x; cur_hz_x = nxt_hz_x; nxt_hz_x = tmp;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < S; ++s) {
      /* pole adjoints from g of the later step, before it is overwritten */
      for (int64_t y = p; y < ny - p + 1; ++y) {
        for (int64_t x = p; x < nx - p + 1; ++x) {
          const int64_t j = y * nx + x, i = s * N + j;
          const REAL gv = lam_ey[i];
          REAL u = (REAL)0;
          for (int64_t pp = 0; pp < NP; ++pp) {
            const int64_t c = pp * N + j, pi = (s * NP + pp) * N + j;
            u = u + db[c] * lpol[pi];
            lpol[pi] = da[c] * lpol[pi] + dcp[c] * gv;
          }
          U[i] = u;
        }
      }
      FN(adj_h)(&g, ca, cq, lam_hx, lam_hz, lam_ey, cur_ey_x, cur_ey_z, nxt_ey_x, nxt_ey_z, s);
      if (A->n_rec > 0)
        FN(inject)(lam_ey, (const REAL *)A->grad_r + t * S * A->n_rec, A->receivers_i,
                   A->n_rec, N, s);
      for (int64_t y = p; y < ny - p + 1; ++y) {
        for (int64_t x = p; x < nx - p + 1; ++x) {
          const int64_t j = y * nx + x, i = s * N + j;
          REAL sb = (REAL)0;
          for (int64_t pp = 0; pp < NP; ++pp)
            sb = sb + db[pp * N + j] * lpol[(s * NP + pp) * N + j];
          lam_ey[i] = (lam_ey[i] + U[i]) + sb;
        }
      }
      if (A->n_src > 0 && A->grad_f)
        FN(record)((REAL *)A->grad_f + t * S * A->n_src, lam_ey, A->sources_i, A->n_src, N, s);
    }
    tmp = cur_ey_x; cur_ey_x = nxt_ey_x; nxt_ey_x = tmp;
    tmp = cur_ey_z; cur_ey_z = nxt_ey_z; nxt_ey_z = tmp;
    ++swaps;
    if ((t % k) != 0) continue;
    const int64_t q = t / k - A->q0;
#pragma omp parallel for schedule(static)
    for (int64_t y = p; y < ny - p + 1; ++y) {
      for (int64_t x = p; x < nx - p + 1; ++x) {
        const int64_t j = y * nx + x;
        /* step-major: the shot terms of each image summed in shot order */
        if (A->grad_ca && A->ey_store) {
          REAL sum = (REAL)0;
          for (int64_t s = 0; s < S; ++s)
            sum = sum + lam_ey[s * N + j] * FN(debye_get)(A->ey_store, bf16, q * SN + s * N + j) *
                            kscale;
          ((REAL *)A->grad_ca)[j] = ((REAL *)A->grad_ca)[j] + sum;
        }
        if (A->grad_cb && A->curl_store) {
          REAL sum = (REAL)0;
          for (int64_t s = 0; s < S; ++s)
            sum = sum + lam_ey[s * N + j] *
                            FN(debye_get)(A->curl_store, bf16, q * SN + s * N + j) * kscale;
          ((REAL *)A->grad_cb)[j] = ((REAL *)A->grad_cb)[j] + sum;
        }
        for (int64_t pp = 0; pp < NP; ++pp) {
          if (A->pol_store && (A->grad_cp || A->grad_a)) {
            REAL scp = (REAL)0, sa = (REAL)0;
            for (int64_t s = 0; s < S; ++s) {
              const REAL pv =
                  FN(debye_get)(A->pol_store, bf16, ((q * S + s) * NP + pp) * N + j);
              scp = scp + lam_ey[s * N + j] * pv * kscale;
              sa = sa + lpol[(s * NP + pp) * N + j] * pv * kscale;
            }
            if (A->grad_cp) ((REAL *)A->grad_cp)[pp * N + j] = ((REAL *)A->grad_cp)[pp * N + j] + scp;
            if (A->grad_a) ((REAL *)A->grad_a)[pp * N + j] = ((REAL *)A->grad_a)[pp * N + j] + sa;
          }
          if (A->esum_store && A->grad_b) {
            REAL sbv = (REAL)0;
            for (int64_t s = 0; s < S; ++s)
              sbv = sbv + lpol[(s * NP + pp) * N + j] *
                              FN(debye_get)(A->esum_store, bf16, q * SN + s * N + j) * kscale;
            ((REAL *)A->grad_b)[pp * N + j] = ((REAL *)A->grad_b)[pp * N + j] + sbv;
          }
        }
      }
    }
  }
  if (swaps % 2 == 1) {
    const size_t nb = (size_t)SN * sizeof(REAL);
    memcpy(A->lam[3], cur_ey_x, nb);
    memcpy(A->lam[4], cur_ey_z, nb);
    memcpy(A->lam[5], cur_hx_z, nb);
    memcpy(A->lam[6], cur_hz_x, nb);
  }
  free(U);
}

#undef FN
#undef CAT2
#undef CAT2_
