/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle for the TM2D time-stepping path.
 *
 * This header is included twice by tm2d_oracle.c, once with REAL=float and
 * once with REAL=double (SFX names the instantiation).  It restates, in plain
 * sequential C, the arithmetic of the reference's TM2D native backend:
 *
 *   forward H half-step   src/tide/csrc/tm2d/maxwell_tm_core.cuh:448-502
 *   forward E half-step   src/tide/csrc/tm2d/maxwell_tm_core.cuh:504-547
 *   E with snapshots      src/tide/csrc/tm2d/maxwell_tm_core.cuh:549-599
 *   sources / receivers   src/tide/csrc/tm2d/maxwell.cu:89-141
 *   exact adjoint E-phase src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:954-1027
 *   exact adjoint H-phase src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1082-1165
 *   coefficient gradient  src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:834-871
 *   reverse time loop     src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:2540-2731
 *   shot reduction        src/tide/csrc/tm2d/maxwell_tm_inst.cpp:2185-2206
 *
 * Every floating-point expression is written in the reference's operation
 * order and the file is compiled without FMA contraction, so the float
 * instantiation reproduces the reference CPU backend's forward bit for bit.
 * The adjoint is the exact transpose used by the reference CUDA backend (the
 * reference CPU backward reuses the forward kernels and is not an exact
 * adjoint for heterogeneous media with CPML).
 *
 * Only the device storage mode (a contiguous [n_store, S, ny, nx] history in
 * the caller's store_1 buffer) is implemented; that is the only mode the
 * oracle is used with.
 */

#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

static REAL FN(coef)(int stencil, int m) {
  switch (stencil) {
  case 2:
    return (REAL)1.0;
  case 4:
    return m == 0 ? (REAL)(9.0 / 8.0) : (REAL)(-1.0 / 24.0);
  case 6:
    return m == 0   ? (REAL)(75.0 / 64.0)
           : m == 1 ? (REAL)(-25.0 / 384.0)
                    : (REAL)(3.0 / 640.0);
  default:
    return m == 0   ? (REAL)(1225.0 / 1024.0)
           : m == 1 ? (REAL)(-245.0 / 3072.0)
           : m == 2 ? (REAL)(49.0 / 5120.0)
                    : (REAL)(-5.0 / 7168.0);
  }
}

/* Forward staggered differences (maxwell_tm_core.cuh:64-190).  For stencil 2
 * the reference omits the unit coefficient; multiplying by 1 is exact, so the
 * generic loop below is bitwise identical. */
static inline REAL FN(d_y1)(const REAL *f, int64_t i, int64_t nx, int st,
                            REAL rd) {
  int p = st / 2;
  REAL acc = FN(coef)(st, 0) * (f[i] - f[i - nx]);
  for (int m = 1; m < p; ++m)
    acc = acc + FN(coef)(st, m) * (f[i + m * nx] - f[i - (m + 1) * nx]);
  return acc * rd;
}
static inline REAL FN(d_x1)(const REAL *f, int64_t i, int st, REAL rd) {
  int p = st / 2;
  REAL acc = FN(coef)(st, 0) * (f[i] - f[i - 1]);
  for (int m = 1; m < p; ++m)
    acc = acc + FN(coef)(st, m) * (f[i + m] - f[i - (m + 1)]);
  return acc * rd;
}
static inline REAL FN(d_yh1)(const REAL *f, int64_t i, int64_t nx, int st,
                             REAL rd) {
  int p = st / 2;
  REAL acc = FN(coef)(st, 0) * (f[i + nx] - f[i]);
  for (int m = 1; m < p; ++m)
    acc = acc + FN(coef)(st, m) * (f[i + (m + 1) * nx] - f[i - m * nx]);
  return acc * rd;
}
static inline REAL FN(d_xh1)(const REAL *f, int64_t i, int st, REAL rd) {
  int p = st / 2;
  REAL acc = FN(coef)(st, 0) * (f[i + 1] - f[i]);
  for (int m = 1; m < p; ++m)
    acc = acc + FN(coef)(st, m) * (f[i + m + 1] - f[i - m]);
  return acc * rd;
}

typedef struct {
  const REAL *ay, *by, *ayh, *byh, *ax, *bx, *axh, *bxh;
  const REAL *ky, *kyh, *kx, *kxh;
  REAL rdy, rdx;
  int64_t n_shots, ny, nx, n_src, n_rec;
  int64_t pml_y0, pml_x0, pml_y1, pml_x1;
  int stencil;
  bool ca_b, cb_b, cq_b;
} FN(geom);

/* H half-step for one shot (maxwell_tm_core.cuh:448-502). */
static void FN(step_h)(const FN(geom) * g, const REAL *cq, const REAL *ey,
                       REAL *hx, REAL *hz, REAL *m_ey_x, REAL *m_ey_z,
                       int64_t s) {
  const int64_t ny = g->ny, nx = g->nx, N = ny * nx;
  const int p = g->stencil / 2;
  const int64_t pml_y1h = g->pml_y1 > g->pml_y0 ? g->pml_y1 - 1 : g->pml_y0;
  const int64_t pml_x1h = g->pml_x1 > g->pml_x0 ? g->pml_x1 - 1 : g->pml_x0;
  for (int64_t y = p; y < ny - p + 1; ++y) {
    for (int64_t x = p; x < nx - p + 1; ++x) {
      const int64_t j = y * nx + x, i = s * N + j;
      const REAL cqv = g->cq_b ? cq[i] : cq[j];
      if (y < ny - p) {
        REAL d = FN(d_yh1)(ey, i, nx, g->stencil, g->rdy);
        if (y < g->pml_y0 || y >= pml_y1h) {
          m_ey_z[i] = g->byh[y] * m_ey_z[i] + g->ayh[y] * d;
          d = d / g->kyh[y] + m_ey_z[i];
        }
        hx[i] -= cqv * d;
      }
      if (x < nx - p) {
        REAL d = FN(d_xh1)(ey, i, g->stencil, g->rdx);
        if (x < g->pml_x0 || x >= pml_x1h) {
          m_ey_x[i] = g->bxh[x] * m_ey_x[i] + g->axh[x] * d;
          d = d / g->kxh[x] + m_ey_x[i];
        }
        hz[i] += cqv * d;
      }
    }
  }
}

static inline uint16_t FN(to_bf16)(REAL v) {
  /* Round-to-nearest-even truncation of an IEEE float (maxwell.cpp:65-75). */
  union {
    float f;
    uint32_t u;
  } t;
  t.f = (float)v;
  uint32_t lsb = (t.u >> 16) & 1u;
  t.u += 0x7FFFu + lsb;
  return (uint16_t)(t.u >> 16);
}
static inline REAL FN(from_bf16)(uint16_t v) {
  union {
    uint32_t u;
    float f;
  } t;
  t.u = ((uint32_t)v) << 16;
  return (REAL)t.f;
}

/* E half-step for one shot (maxwell_tm_core.cuh:504-599).  When a store
 * pointer is given, Ey^n and curl H^n are written before the update. */
static void FN(step_e)(const FN(geom) * g, const REAL *ca, const REAL *cb,
                       const REAL *hx, const REAL *hz, REAL *ey, REAL *m_hx_z,
                       REAL *m_hz_x, void *ey_store, void *curl_store,
                       bool bf16, int64_t s) {
  const int64_t ny = g->ny, nx = g->nx, N = ny * nx;
  const int p = g->stencil / 2;
  for (int64_t y = p; y < ny - p + 1; ++y) {
    for (int64_t x = p; x < nx - p + 1; ++x) {
      const int64_t j = y * nx + x, i = s * N + j;
      const REAL cav = g->ca_b ? ca[i] : ca[j];
      const REAL cbv = g->cb_b ? cb[i] : cb[j];
      REAL dhz_dx = FN(d_x1)(hz, i, g->stencil, g->rdx);
      REAL dhx_dz = FN(d_y1)(hx, i, nx, g->stencil, g->rdy);
      if (x < g->pml_x0 || x >= g->pml_x1) {
        m_hz_x[i] = g->bx[x] * m_hz_x[i] + g->ax[x] * dhz_dx;
        dhz_dx = dhz_dx / g->kx[x] + m_hz_x[i];
      }
      if (y < g->pml_y0 || y >= g->pml_y1) {
        m_hx_z[i] = g->by[y] * m_hx_z[i] + g->ay[y] * dhx_dz;
        dhx_dz = dhx_dz / g->ky[y] + m_hx_z[i];
      }
      const REAL curl = dhz_dx - dhx_dz;
      if (ey_store) {
        if (bf16)
          ((uint16_t *)ey_store)[i] = FN(to_bf16)(ey[i]);
        else
          ((REAL *)ey_store)[i] = ey[i];
      }
      if (curl_store) {
        if (bf16)
          ((uint16_t *)curl_store)[i] = FN(to_bf16)(curl);
        else
          ((REAL *)curl_store)[i] = curl;
      }
      ey[i] = cav * ey[i] + cbv * curl;
    }
  }
}

/* Born E half-step for one shot (maxwell_tm_core.cuh:601-690): background
 * and scattered curls with their own CPML memories; the scattered update adds
 * dca Ey^n + dcb curl H^n of the background. */
static void FN(step_e_born)(const FN(geom) * g, const REAL *ca, const REAL *cb,
                            const REAL *dca, const REAL *dcb, const REAL *hx,
                            const REAL *hz, REAL *ey, REAL *m_hx_z,
                            REAL *m_hz_x, const REAL *dhx, const REAL *dhz,
                            REAL *dey, REAL *dm_hx_z, REAL *dm_hz_x,
                            void *const st[4], bool bf16, int64_t s) {
  const int64_t ny = g->ny, nx = g->nx, N = ny * nx;
  const int p = g->stencil / 2;
  for (int64_t y = p; y < ny - p + 1; ++y) {
    for (int64_t x = p; x < nx - p + 1; ++x) {
      const int64_t j = y * nx + x, i = s * N + j;
      const REAL cav = g->ca_b ? ca[i] : ca[j];
      const REAL cbv = g->cb_b ? cb[i] : cb[j];
      const REAL dcav = g->ca_b ? dca[i] : dca[j];
      const REAL dcbv = g->cb_b ? dcb[i] : dcb[j];
      const bool pml_x = x < g->pml_x0 || x >= g->pml_x1;
      const bool pml_y = y < g->pml_y0 || y >= g->pml_y1;
      REAL dhz_dx = FN(d_x1)(hz, i, g->stencil, g->rdx);
      REAL dhx_dz = FN(d_y1)(hx, i, nx, g->stencil, g->rdy);
      if (pml_x) {
        m_hz_x[i] = g->bx[x] * m_hz_x[i] + g->ax[x] * dhz_dx;
        dhz_dx = dhz_dx / g->kx[x] + m_hz_x[i];
      }
      if (pml_y) {
        m_hx_z[i] = g->by[y] * m_hx_z[i] + g->ay[y] * dhx_dz;
        dhx_dz = dhx_dz / g->ky[y] + m_hx_z[i];
      }
      const REAL curl = dhz_dx - dhx_dz;
      REAL ddhz_dx = FN(d_x1)(dhz, i, g->stencil, g->rdx);
      REAL ddhx_dz = FN(d_y1)(dhx, i, nx, g->stencil, g->rdy);
      if (pml_x) {
        dm_hz_x[i] = g->bx[x] * dm_hz_x[i] + g->ax[x] * ddhz_dx;
        ddhz_dx = ddhz_dx / g->kx[x] + dm_hz_x[i];
      }
      if (pml_y) {
        dm_hx_z[i] = g->by[y] * dm_hx_z[i] + g->ay[y] * ddhx_dz;
        ddhx_dz = ddhx_dz / g->ky[y] + dm_hx_z[i];
      }
      const REAL dcurl = ddhz_dx - ddhx_dz;
      const REAL ey_n = ey[i], dey_n = dey[i];
      /* snapshots before the update: Ey^n, curl H^n, dEy^n, dcurl */
      const REAL vals[4] = {ey_n, curl, dey_n, dcurl};
      for (int k = 0; k < 4; ++k)
        if (st && st[k]) {
          if (bf16)
            ((uint16_t *)st[k])[i] = FN(to_bf16)(vals[k]);
          else
            ((REAL *)st[k])[i] = vals[k];
        }
      ey[i] = cav * ey_n + cbv * curl;
      dey[i] = cav * dey_n + cbv * dcurl + dcav * ey_n + dcbv * curl;
    }
  }
}

/* ---------------- exact adjoint (maxwell_tm_cuda_inst.cu:954-1165) -------- */

static inline REAL FN(raw_x)(const FN(geom) * g, const REAL *cb,
                             const REAL *lam_ey, const REAL *m_hz_x,
                             int64_t base, int64_t y, int64_t x) {
  const int p = g->stencil / 2;
  if (y < p || y >= g->ny - p + 1 || x < p || x >= g->nx - p + 1)
    return (REAL)0;
  const int64_t j = y * g->nx + x, i = base + j;
  const REAL q = (g->cb_b ? cb[i] : cb[j]) * lam_ey[i];
  if (x >= g->pml_x0 && x < g->pml_x1)
    return q;
  const REAL m_next = g->bx[x] * m_hz_x[i] + q;
  return g->ax[x] * m_next + q / g->kx[x];
}

static inline REAL FN(raw_y)(const FN(geom) * g, const REAL *cb,
                             const REAL *lam_ey, const REAL *m_hx_z,
                             int64_t base, int64_t y, int64_t x) {
  const int p = g->stencil / 2;
  if (y < p || y >= g->ny - p + 1 || x < p || x >= g->nx - p + 1)
    return (REAL)0;
  const int64_t j = y * g->nx + x, i = base + j;
  const REAL q = (g->cb_b ? cb[i] : cb[j]) * lam_ey[i];
  if (y >= g->pml_y0 && y < g->pml_y1)
    return -q;
  const REAL m_next = g->by[y] * m_hx_z[i] - q;
  return g->ay[y] * m_next - q / g->ky[y];
}

static void FN(adj_e)(const FN(geom) * g, const REAL *cb, const REAL *lam_ey,
                      REAL *lam_hx, REAL *lam_hz, const REAL *m_hx_z,
                      const REAL *m_hz_x, REAL *m_hx_z_n, REAL *m_hz_x_n,
                      int64_t s) {
  const int64_t ny = g->ny, nx = g->nx, N = ny * nx, base = s * N;
  const int p = g->stencil / 2;
  const int st = g->stencil;
  for (int64_t y = p; y < ny - p + 1; ++y) {
    for (int64_t x = p; x < nx - p + 1; ++x) {
      const int64_t j = y * nx + x, i = base + j;
      const REAL q = (g->cb_b ? cb[i] : cb[j]) * lam_ey[i];
      const bool px = x < g->pml_x0 || x >= g->pml_x1;
      const bool py = y < g->pml_y0 || y >= g->pml_y1;
      m_hz_x_n[i] = px ? g->bx[x] * m_hz_x[i] + q : (REAL)0;
      m_hx_z_n[i] = py ? g->by[y] * m_hx_z[i] - q : (REAL)0;
      /* diff_x1_adj: sum_m c_m (raw(x-m) - raw(x+1+m)) * rdx */
      REAL ax_ = FN(coef)(st, 0) *
                 (FN(raw_x)(g, cb, lam_ey, m_hz_x, base, y, x) -
                  FN(raw_x)(g, cb, lam_ey, m_hz_x, base, y, x + 1));
      for (int m = 1; m < p; ++m)
        ax_ = ax_ + FN(coef)(st, m) *
                        (FN(raw_x)(g, cb, lam_ey, m_hz_x, base, y, x - m) -
                         FN(raw_x)(g, cb, lam_ey, m_hz_x, base, y, x + 1 + m));
      lam_hz[i] += ax_ * g->rdx;
      REAL ay_ = FN(coef)(st, 0) *
                 (FN(raw_y)(g, cb, lam_ey, m_hx_z, base, y, x) -
                  FN(raw_y)(g, cb, lam_ey, m_hx_z, base, y + 1, x));
      for (int m = 1; m < p; ++m)
        ay_ = ay_ + FN(coef)(st, m) *
                        (FN(raw_y)(g, cb, lam_ey, m_hx_z, base, y - m, x) -
                         FN(raw_y)(g, cb, lam_ey, m_hx_z, base, y + 1 + m, x));
      lam_hx[i] += ay_ * g->rdy;
    }
  }
}

static inline REAL FN(raw_eyz)(const FN(geom) * g, const REAL *cq,
                               const REAL *lam_hx, const REAL *m_ey_z,
                               int64_t base, int64_t y, int64_t x,
                               int64_t pml_y1h) {
  const int p = g->stencil / 2;
  if (y < p || y >= g->ny - p || x < p || x >= g->nx - p + 1)
    return (REAL)0;
  const int64_t j = y * g->nx + x, i = base + j;
  const REAL adj = -(g->cq_b ? cq[i] : cq[j]) * lam_hx[i];
  if (y >= g->pml_y0 && y < pml_y1h)
    return adj;
  const REAL m_next = g->byh[y] * m_ey_z[i] + adj;
  return g->ayh[y] * m_next + adj / g->kyh[y];
}

static inline REAL FN(raw_eyx)(const FN(geom) * g, const REAL *cq,
                               const REAL *lam_hz, const REAL *m_ey_x,
                               int64_t base, int64_t y, int64_t x,
                               int64_t pml_x1h) {
  const int p = g->stencil / 2;
  if (y < p || y >= g->ny - p + 1 || x < p || x >= g->nx - p)
    return (REAL)0;
  const int64_t j = y * g->nx + x, i = base + j;
  const REAL adj = (g->cq_b ? cq[i] : cq[j]) * lam_hz[i];
  if (x >= g->pml_x0 && x < pml_x1h)
    return adj;
  const REAL m_next = g->bxh[x] * m_ey_x[i] + adj;
  return g->axh[x] * m_next + adj / g->kxh[x];
}

static void FN(adj_h)(const FN(geom) * g, const REAL *ca, const REAL *cq,
                      const REAL *lam_hx, const REAL *lam_hz, REAL *lam_ey,
                      const REAL *m_ey_x, const REAL *m_ey_z, REAL *m_ey_x_n,
                      REAL *m_ey_z_n, int64_t s) {
  const int64_t ny = g->ny, nx = g->nx, N = ny * nx, base = s * N;
  const int p = g->stencil / 2;
  const int st = g->stencil;
  const int64_t pml_y1h = g->pml_y1 > g->pml_y0 ? g->pml_y1 - 1 : g->pml_y0;
  const int64_t pml_x1h = g->pml_x1 > g->pml_x0 ? g->pml_x1 - 1 : g->pml_x0;
  for (int64_t y = p; y < ny - p + 1; ++y) {
    for (int64_t x = p; x < nx - p + 1; ++x) {
      const int64_t j = y * nx + x, i = base + j;
      const REAL cqv = g->cq_b ? cq[i] : cq[j];
      const bool py = y < g->pml_y0 || y >= pml_y1h;
      const bool px = x < g->pml_x0 || x >= pml_x1h;
      const REAL adj_y = -cqv * lam_hx[i];
      const REAL adj_x = cqv * lam_hz[i];
      m_ey_z_n[i] = (y < ny - p && py) ? g->byh[y] * m_ey_z[i] + adj_y : (REAL)0;
      m_ey_x_n[i] = (x < nx - p && px) ? g->bxh[x] * m_ey_x[i] + adj_x : (REAL)0;
      const REAL cav = g->ca_b ? ca[i] : ca[j];
      lam_ey[i] = cav * lam_ey[i];
      /* diff_yh1_adj: sum_m c_m (raw(y-1-m) - raw(y+m)) * rdy */
      REAL dz = FN(coef)(st, 0) *
                (FN(raw_eyz)(g, cq, lam_hx, m_ey_z, base, y - 1, x, pml_y1h) -
                 FN(raw_eyz)(g, cq, lam_hx, m_ey_z, base, y, x, pml_y1h));
      for (int m = 1; m < p; ++m)
        dz = dz + FN(coef)(st, m) *
                      (FN(raw_eyz)(g, cq, lam_hx, m_ey_z, base, y - 1 - m, x,
                                   pml_y1h) -
                       FN(raw_eyz)(g, cq, lam_hx, m_ey_z, base, y + m, x,
                                   pml_y1h));
      REAL dx = FN(coef)(st, 0) *
                (FN(raw_eyx)(g, cq, lam_hz, m_ey_x, base, y, x - 1, pml_x1h) -
                 FN(raw_eyx)(g, cq, lam_hz, m_ey_x, base, y, x, pml_x1h));
      for (int m = 1; m < p; ++m)
        dx = dx + FN(coef)(st, m) *
                      (FN(raw_eyx)(g, cq, lam_hz, m_ey_x, base, y, x - 1 - m,
                                   pml_x1h) -
                       FN(raw_eyx)(g, cq, lam_hz, m_ey_x, base, y, x + m,
                                   pml_x1h));
      lam_ey[i] += dz * g->rdy + dx * g->rdx;
    }
  }
}

static void FN(inject)(REAL *field, const REAL *vals, const int64_t *idx,
                       int64_t n_per_shot, int64_t N, int64_t s) {
  for (int64_t k = 0; k < n_per_shot; ++k) {
    const int64_t e = s * n_per_shot + k;
    if (idx[e] >= 0)
      field[s * N + idx[e]] += vals[e];
  }
}
static void FN(record)(REAL *out, const REAL *field, const int64_t *idx,
                       int64_t n_per_shot, int64_t N, int64_t s) {
  for (int64_t k = 0; k < n_per_shot; ++k) {
    const int64_t e = s * n_per_shot + k;
    if (idx[e] >= 0)
      out[e] = field[s * N + idx[e]];
  }
}

#define ORACLE_GEOM_INIT                                                       \
  FN(geom) g;                                                                  \
  g.ay = ay; g.by = by; g.ayh = ayh; g.byh = byh;                              \
  g.ax = ax; g.bx = bx; g.axh = axh; g.bxh = bxh;                              \
  g.ky = ky; g.kyh = kyh; g.kx = kx; g.kxh = kxh;                              \
  g.rdy = rdy; g.rdx = rdx; g.n_shots = n_shots; g.ny = ny; g.nx = nx;         \
  g.n_src = n_src; g.n_rec = n_rec; g.pml_y0 = pml_y0; g.pml_x0 = pml_x0;      \
  g.pml_y1 = pml_y1; g.pml_x1 = pml_x1; g.stencil = stencil;                   \
  g.ca_b = ca_batched; g.cb_b = cb_batched; g.cq_b = cq_batched;

/* Forward without storage: same argument meaning as the reference's
 * maxwell_tm_{S}_{dtype}_forward (maxwell_tm_inst.cpp:734-818).  Debye
 * dispersion is handled by the tm2d Debye oracle instead. */
void FN(tide_oracle_tm_forward)(
    int stencil, const REAL *ca, const REAL *cb, const REAL *cq, const REAL *f,
    REAL *ey, REAL *hx, REAL *hz, REAL *m_ey_x, REAL *m_ey_z, REAL *m_hx_z,
    REAL *m_hz_x, REAL *r, const REAL *ay, const REAL *by, const REAL *ayh,
    const REAL *byh, const REAL *ax, const REAL *bx, const REAL *axh,
    const REAL *bxh, const REAL *ky, const REAL *kyh, const REAL *kx,
    const REAL *kxh, const int64_t *sources_i, const int64_t *receivers_i,
    REAL rdy, REAL rdx, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx,
    int64_t n_src, int64_t n_rec, bool ca_batched, bool cb_batched,
    bool cq_batched, int64_t start_t, int64_t pml_y0, int64_t pml_x0,
    int64_t pml_y1, int64_t pml_x1) {
  ORACLE_GEOM_INIT
  const int64_t N = ny * nx;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < n_shots; ++s) {
    for (int64_t t = start_t; t < start_t + nt; ++t) {
      FN(step_h)(&g, cq, ey, hx, hz, m_ey_x, m_ey_z, s);
      FN(step_e)(&g, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, NULL, NULL, false, s);
      if (n_src > 0)
        FN(inject)(ey, f + t * n_shots * n_src, sources_i, n_src, N, s);
      if (n_rec > 0)
        FN(record)(r + t * n_shots * n_rec, ey, receivers_i, n_rec, N, s);
    }
  }
}

/* Forward with snapshot storage in a device-mode history [n_store,S,ny,nx]
 * (maxwell_tm_inst.cpp:833-955).  storage_format 1 stores bf16. */
void FN(tide_oracle_tm_forward_with_storage)(
    int stencil, const REAL *ca, const REAL *cb, const REAL *cq, const REAL *f,
    REAL *ey, REAL *hx, REAL *hz, REAL *m_ey_x, REAL *m_ey_z, REAL *m_hx_z,
    REAL *m_hz_x, REAL *r, void *ey_store, void *curl_store, const REAL *ay,
    const REAL *by, const REAL *ayh, const REAL *byh, const REAL *ax,
    const REAL *bx, const REAL *axh, const REAL *bxh, const REAL *ky,
    const REAL *kyh, const REAL *kx, const REAL *kxh, const int64_t *sources_i,
    const int64_t *receivers_i, REAL rdy, REAL rdx, int64_t nt,
    int64_t n_shots, int64_t ny, int64_t nx, int64_t n_src, int64_t n_rec,
    int64_t step_ratio, int64_t storage_format, bool ca_requires_grad,
    bool cb_requires_grad, bool ca_batched, bool cb_batched, bool cq_batched,
    int64_t start_t, int64_t pml_y0, int64_t pml_x0, int64_t pml_y1,
    int64_t pml_x1) {
  ORACLE_GEOM_INIT
  const int64_t N = ny * nx;
  const bool bf16 = storage_format == 1;
  const size_t esz = bf16 ? 2 : sizeof(REAL);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < n_shots; ++s) {
    for (int64_t t = start_t; t < start_t + nt; ++t) {
      FN(step_h)(&g, cq, ey, hx, hz, m_ey_x, m_ey_z, s);
      const bool store = (t % step_ratio) == 0;
      const int64_t off = (t / step_ratio) * n_shots * N;
      void *es = (store && ca_requires_grad && ey_store)
                     ? (void *)((char *)ey_store + (size_t)off * esz)
                     : NULL;
      void *cs = (store && cb_requires_grad && curl_store)
                     ? (void *)((char *)curl_store + (size_t)off * esz)
                     : NULL;
      FN(step_e)(&g, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, es, cs, bf16, s);
      if (n_src > 0)
        FN(inject)(ey, f + t * n_shots * n_src, sources_i, n_src, N, s);
      if (n_rec > 0)
        FN(record)(r + t * n_shots * n_rec, ey, receivers_i, n_rec, N, s);
    }
  }
}

/* Born forward: argument meaning of the reference's
 * maxwell_tm_{S}_{dtype}_born_forward (maxwell_tm_inst.cpp:962-1045); with
 * store (4 histories [n_store, S, ny, nx]: background Ey^n, curl H^n,
 * scattered dEy^n, dcurl; NULL entries are skipped) the snapshots of steps
 * t % step_ratio == 0 into slot t / step_ratio. */
void FN(tide_oracle_tm_born_forward_store)(
    int stencil, const REAL *ca, const REAL *cb, const REAL *cq,
    const REAL *dca, const REAL *dcb, const REAL *f0, const REAL *df,
    REAL *ey, REAL *hx, REAL *hz, REAL *m_ey_x, REAL *m_ey_z, REAL *m_hx_z,
    REAL *m_hz_x, REAL *dey, REAL *dhx, REAL *dhz, REAL *dm_ey_x,
    REAL *dm_ey_z, REAL *dm_hx_z, REAL *dm_hz_x, REAL *r, REAL *background_r,
    const REAL *ay, const REAL *by, const REAL *ayh, const REAL *byh,
    const REAL *ax, const REAL *bx, const REAL *axh, const REAL *bxh,
    const REAL *ky, const REAL *kyh, const REAL *kx, const REAL *kxh,
    const int64_t *sources_i, const int64_t *receivers_i, REAL rdy, REAL rdx,
    int64_t nt, int64_t n_shots, int64_t ny, int64_t nx, int64_t n_src,
    int64_t n_rec, bool ca_batched, bool cb_batched, bool cq_batched,
    int64_t start_t, int64_t pml_y0, int64_t pml_x0, int64_t pml_y1,
    int64_t pml_x1, void **store, int64_t step_ratio, int64_t storage_format) {
  ORACLE_GEOM_INIT
  const int64_t N = ny * nx;
  const bool bf16 = storage_format == 1;
  const size_t esz = bf16 ? 2 : sizeof(REAL);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < n_shots; ++s) {
    for (int64_t t = start_t; t < start_t + nt; ++t) {
      FN(step_h)(&g, cq, ey, hx, hz, m_ey_x, m_ey_z, s);
      FN(step_h)(&g, cq, dey, dhx, dhz, dm_ey_x, dm_ey_z, s);
      void *st[4] = {NULL, NULL, NULL, NULL};
      if (store && step_ratio > 0 && t % step_ratio == 0)
        for (int k = 0; k < 4; ++k)
          if (store[k])
            st[k] = (char *)store[k] + (size_t)((t / step_ratio) * n_shots * N) * esz;
      FN(step_e_born)(&g, ca, cb, dca, dcb, hx, hz, ey, m_hx_z, m_hz_x, dhx,
                      dhz, dey, dm_hx_z, dm_hz_x, st, bf16, s);
      if (n_src > 0) {
        FN(inject)(ey, f0 + t * n_shots * n_src, sources_i, n_src, N, s);
        FN(inject)(dey, df + t * n_shots * n_src, sources_i, n_src, N, s);
      }
      if (n_rec > 0) {
        FN(record)(r + t * n_shots * n_rec, dey, receivers_i, n_rec, N, s);
        if (background_r)
          FN(record)(background_r + t * n_shots * n_rec, ey, receivers_i,
                     n_rec, N, s);
      }
    }
  }
}

void FN(tide_oracle_tm_born_forward)(
    int stencil, const REAL *ca, const REAL *cb, const REAL *cq,
    const REAL *dca, const REAL *dcb, const REAL *f0, const REAL *df,
    REAL *ey, REAL *hx, REAL *hz, REAL *m_ey_x, REAL *m_ey_z, REAL *m_hx_z,
    REAL *m_hz_x, REAL *dey, REAL *dhx, REAL *dhz, REAL *dm_ey_x,
    REAL *dm_ey_z, REAL *dm_hx_z, REAL *dm_hz_x, REAL *r, REAL *background_r,
    const REAL *ay, const REAL *by, const REAL *ayh, const REAL *byh,
    const REAL *ax, const REAL *bx, const REAL *axh, const REAL *bxh,
    const REAL *ky, const REAL *kyh, const REAL *kx, const REAL *kxh,
    const int64_t *sources_i, const int64_t *receivers_i, REAL rdy, REAL rdx,
    int64_t nt, int64_t n_shots, int64_t ny, int64_t nx, int64_t n_src,
    int64_t n_rec, bool ca_batched, bool cb_batched, bool cq_batched,
    int64_t start_t, int64_t pml_y0, int64_t pml_x0, int64_t pml_y1,
    int64_t pml_x1) {
  FN(tide_oracle_tm_born_forward_store)(
      stencil, ca, cb, cq, dca, dcb, f0, df, ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x, dey,
      dhx, dhz, dm_ey_x, dm_ey_z, dm_hx_z, dm_hz_x, r, background_r, ay, by, ayh, byh, ax, bx,
      axh, bxh, ky, kyh, kx, kxh, sources_i, receivers_i, rdy, rdx, nt, n_shots, ny, nx, n_src,
      n_rec, ca_batched, cb_batched, cq_batched, start_t, pml_y0, pml_x0, pml_y1, pml_x1, NULL,
      0, 0);
}

/* Exact adjoint with fused coefficient gradient, device storage mode.
 * Interface semantics follow the reference CPU backward
 * (maxwell_tm_inst.cpp:1997-2219: batched models accumulate straight into
 * grad_ca/grad_cb); arithmetic follows the reference CUDA exact adjoint
 * (maxwell_tm_cuda_inst.cu:2405-2734).  adjoint_memory_scratch holds the four
 * next-step adjoint memories.
 *
 * The shot reduction of the model gradient has two summation orders
 * (tide_oracle_set_grad_order):
 *   0 (default) the reference's: per-shot accumulators over time, then a sum
 *     over shots at the end (maxwell_tm_inst.cpp:2185-2206);
 *   1 step-major: at every imaged step the shot terms are summed in shot order
 *     and added to the model gradient (the order the CUDA kernels use).
 * Both are exact sums of the same terms; they differ only in rounding. */
void FN(tide_oracle_tm_backward)(
    int stencil, const REAL *ca, const REAL *cb, const REAL *cq,
    const REAL *grad_r, REAL *lam_ey, REAL *lam_hx, REAL *lam_hz,
    REAL *m_lam_ey_x, REAL *m_lam_ey_z, REAL *m_lam_hx_z, REAL *m_lam_hz_x,
    REAL *scratch, const void *ey_store, const void *curl_store, REAL *grad_f,
    REAL *grad_ca, REAL *grad_cb, REAL *grad_ca_shot, REAL *grad_cb_shot,
    const REAL *ay, const REAL *by, const REAL *ayh, const REAL *byh,
    const REAL *ax, const REAL *bx, const REAL *axh, const REAL *bxh,
    const REAL *ky, const REAL *kyh, const REAL *kx, const REAL *kxh,
    const int64_t *sources_i, const int64_t *receivers_i, REAL rdy, REAL rdx,
    int64_t nt, int64_t n_shots, int64_t ny, int64_t nx, int64_t n_src,
    int64_t n_rec, int64_t step_ratio, int64_t storage_format,
    bool ca_requires_grad, bool cb_requires_grad, bool ca_batched,
    bool cb_batched, bool cq_batched, int64_t start_t, int64_t pml_y0,
    int64_t pml_x0, int64_t pml_y1, int64_t pml_x1) {
  ORACLE_GEOM_INIT
  const int64_t N = ny * nx, SN = n_shots * N;
  const int p = stencil / 2;
  const bool bf16 = storage_format == 1;
  const bool step_major = g_oracle_grad_order == 1;
  REAL *acc_ca = ca_batched ? grad_ca : grad_ca_shot;
  REAL *acc_cb = cb_batched ? grad_cb : grad_cb_shot;
  if (ca_requires_grad && !ca_batched)
    memset(grad_ca_shot, 0, (size_t)SN * sizeof(REAL));
  if (cb_requires_grad && !cb_batched)
    memset(grad_cb_shot, 0, (size_t)SN * sizeof(REAL));
  memset(scratch, 0, (size_t)4 * SN * sizeof(REAL));
  const REAL kscale = (REAL)step_ratio;
  REAL *cur_ey_x = m_lam_ey_x, *cur_ey_z = m_lam_ey_z;
  REAL *cur_hx_z = m_lam_hx_z, *cur_hz_x = m_lam_hz_x;
  REAL *nxt_ey_x = scratch, *nxt_ey_z = scratch + SN;
  REAL *nxt_hx_z = scratch + 2 * SN, *nxt_hz_x = scratch + 3 * SN;
  int64_t swaps = 0;
  for (int64_t t = start_t - 1; t >= start_t - nt; --t) {
    REAL *tmp;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < n_shots; ++s)
      FN(adj_e)(&g, cb, lam_ey, lam_hx, lam_hz, cur_hx_z, cur_hz_x, nxt_hx_z,
                nxt_hz_x, s);
    tmp = cur_hx_z; cur_hx_z = nxt_hx_z; nxt_hx_z = tmp;
    tmp = cur_hz_x; cur_hz_x = nxt_hz_x; nxt_hz_x = tmp;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < n_shots; ++s) {
      FN(adj_h)(&g, ca, cq, lam_hx, lam_hz, lam_ey, cur_ey_x, cur_ey_z,
                nxt_ey_x, nxt_ey_z, s);
      if (n_rec > 0)
        FN(inject)(lam_ey, grad_r + t * n_shots * n_rec, receivers_i, n_rec, N,
                   s);
      if (n_src > 0)
        FN(record)(grad_f + t * n_shots * n_src, lam_ey, sources_i, n_src, N,
                   s);
    }
    tmp = cur_ey_x; cur_ey_x = nxt_ey_x; nxt_ey_x = tmp;
    tmp = cur_ey_z; cur_ey_z = nxt_ey_z; nxt_ey_z = tmp;
    ++swaps;
    if ((t % step_ratio) != 0 || !(ca_requires_grad || cb_requires_grad))
      continue;
    const int64_t off = (t / step_ratio) * SN;
#pragma omp parallel for schedule(static)
    for (int64_t y = p; y < ny - p + 1; ++y) {
      for (int64_t x = p; x < nx - p + 1; ++x) {
        const int64_t j = y * nx + x;
        for (int pass = 0; pass < 2; ++pass) {
          const bool want = pass == 0 ? ca_requires_grad : cb_requires_grad;
          if (!want)
            continue;
          const void *store = pass == 0 ? ey_store : curl_store;
          const bool batched = pass == 0 ? ca_batched : cb_batched;
          REAL *acc = pass == 0 ? acc_ca : acc_cb;
          REAL *grad = pass == 0 ? grad_ca : grad_cb;
          REAL sum = (REAL)0;
          for (int64_t s = 0; s < n_shots; ++s) {
            const int64_t i = s * N + j;
            const REAL v = bf16 ? FN(from_bf16)(((const uint16_t *)store)[off + i])
                                : ((const REAL *)store)[off + i];
            const REAL term = lam_ey[i] * v * kscale;
            if (batched || !step_major)
              acc[i] += term;
            else
              sum = sum + term;
          }
          if (step_major && !batched)
            grad[j] = grad[j] + sum;
        }
      }
    }
  }
  /* Leave the final adjoint memories in the caller's arrays. */
  if (swaps % 2 == 1) {
    const size_t nb = (size_t)SN * sizeof(REAL);
    memcpy(m_lam_ey_x, cur_ey_x, nb);
    memcpy(m_lam_ey_z, cur_ey_z, nb);
    memcpy(m_lam_hx_z, cur_hx_z, nb);
    memcpy(m_lam_hz_x, cur_hz_x, nb);
  }
  if (step_major)
    return;
  for (int pass = 0; pass < 2; ++pass) {
    const bool want = pass == 0 ? (ca_requires_grad && !ca_batched)
                                : (cb_requires_grad && !cb_batched);
    REAL *grad = pass == 0 ? grad_ca : grad_cb;
    const REAL *shot = pass == 0 ? grad_ca_shot : grad_cb_shot;
    if (!want)
      continue;
    for (int64_t y = p; y < ny - p + 1; ++y) {
      for (int64_t x = p; x < nx - p + 1; ++x) {
        const int64_t j = y * nx + x;
        REAL sum = (REAL)0;
        for (int64_t s = 0; s < n_shots; ++s)
          sum += shot[s * N + j];
        grad[j] += sum;
      }
    }
  }
}

/* Step-major image of one stored step: grad[j] += sum over shots, in shot
 * order, of lam[s, j] * store[s, j] * k (cells of the update domain). */
static void FN(image_step)(const FN(geom) * g, const REAL *lam, const void *store, int64_t off,
                           int bf16, REAL kscale, REAL *grad, int batched) {
  const int64_t N = g->ny * g->nx;
  const int p = g->stencil / 2;
  for (int64_t y = p; y < g->ny - p + 1; ++y)
    for (int64_t x = p; x < g->nx - p + 1; ++x) {
      const int64_t j = y * g->nx + x;
      REAL sum = (REAL)0;
      for (int64_t s = 0; s < g->n_shots; ++s) {
        const int64_t i = s * N + j;
        const REAL v = bf16 ? FN(from_bf16)(((const uint16_t *)store)[off + i])
                            : ((const REAL *)store)[off + i];
        const REAL term = lam[i] * v * kscale;
        if (batched)
          grad[i] = grad[i] + term;
        else
          sum = sum + term;
      }
      if (!batched) grad[j] = grad[j] + sum;
    }
}

/* Derivative of the Born receivers (and of the background receivers) in the
 * background model, the perturbation and both source terms: the exact adjoint
 * of the joint background + scattered recurrence (the reference's
 * born_backward_bggrad, maxwell_tm_cuda_inst.cu:2785-3200, in its own
 * formulation).  lam is the scattered state's adjoint (driven by grad_r),
 * eta the background's (driven by grad_bg_r and by the scattered update's
 * dependence on the background, dE' += dca E + dcb curlH):
 *   per step, with lam and eta at t+1:  W = cb eta + dcb lam (the curl-H
 *   adjoint's source of the background), eta_Ey <- ca eta + dca lam; the E-
 *   and H-phase adjoints of lam (cb, ca) and of eta (with W in place of
 *   cb eta and unit ca); receivers grad_r -> lam, grad_bg_r -> eta; sources
 *   grad_df <- lam, grad_f0 <- eta; at stored steps, step-major:
 *   grad_ca += eta E + lam dE,  grad_cb += eta curlH + lam dcurl,
 *   grad_dca += lam E,  grad_dcb += lam curlH  (each times k, in that order).
 * Stores: [n_store, S, ny, nx] background Ey / curl H and scattered dEy /
 * dcurl.  scratch: 8 S ny nx (next-step memories of lam then eta). */
void FN(tide_oracle_tm_born_bggrad)(
    int stencil, const REAL *ca, const REAL *cb, const REAL *cq, const REAL *dca,
    const REAL *dcb, const REAL *grad_r, const REAL *grad_bg_r, REAL *lam_ey, REAL *lam_hx,
    REAL *lam_hz, REAL **m_lam, REAL *eta_ey, REAL *eta_hx, REAL *eta_hz, REAL **m_eta,
    REAL *scratch, const void *ey_store, const void *curl_store, const void *dey_store,
    const void *dcurl_store, REAL *grad_df, REAL *grad_f0, REAL *grad_ca, REAL *grad_cb,
    REAL *grad_dca, REAL *grad_dcb, const REAL *ay, const REAL *by, const REAL *ayh,
    const REAL *byh, const REAL *ax, const REAL *bx, const REAL *axh, const REAL *bxh,
    const REAL *ky, const REAL *kyh, const REAL *kx, const REAL *kxh,
    const int64_t *sources_i, const int64_t *receivers_i, REAL rdy, REAL rdx, int64_t nt,
    int64_t n_shots, int64_t ny, int64_t nx, int64_t n_src, int64_t n_rec,
    int64_t step_ratio, int64_t storage_format, bool ca_batched, bool cb_batched,
    bool cq_batched, int64_t start_t, int64_t pml_y0, int64_t pml_x0, int64_t pml_y1,
    int64_t pml_x1) {
  ORACLE_GEOM_INIT
  const int64_t N = ny * nx, SN = n_shots * N;
  const int p = stencil / 2;
  const int bf16 = storage_format == 1;
  const REAL kscale = (REAL)step_ratio;
  REAL *ones = (REAL *)malloc((size_t)SN * sizeof(REAL));
  REAL *w = (REAL *)calloc((size_t)SN, sizeof(REAL));
  for (int64_t i = 0; i < SN; ++i) ones[i] = (REAL)1;
  memset(scratch, 0, (size_t)8 * SN * sizeof(REAL));
  /* memories: 0 ey_x, 1 ey_z, 2 hx_z, 3 hz_x; cur / next per state */
  REAL *cl[4], *nl[4], *ce[4], *ne[4];
  for (int m = 0; m < 4; ++m) {
    cl[m] = m_lam[m];
    nl[m] = scratch + m * SN;
    ce[m] = m_eta[m];
    ne[m] = scratch + (4 + m) * SN;
  }
  int64_t swaps = 0;
  for (int64_t t = start_t - 1; t >= start_t - nt; --t) {
    REAL *tmp;
    for (int64_t s = 0; s < n_shots; ++s)
      for (int64_t y = p; y < ny - p + 1; ++y)
        for (int64_t x = p; x < nx - p + 1; ++x) {
          const int64_t j = y * nx + x, i = s * N + j;
          const REAL cbv = cb_batched ? cb[i] : cb[j], dcbv = cb_batched ? dcb[i] : dcb[j];
          const REAL cav = ca_batched ? ca[i] : ca[j], dcav = ca_batched ? dca[i] : dca[j];
          w[i] = cbv * eta_ey[i] + dcbv * lam_ey[i];
          eta_ey[i] = cav * eta_ey[i] + dcav * lam_ey[i];
        }
    for (int64_t s = 0; s < n_shots; ++s) {
      FN(adj_e)(&g, cb, lam_ey, lam_hx, lam_hz, cl[2], cl[3], nl[2], nl[3], s);
      FN(adj_e)(&g, ones, w, eta_hx, eta_hz, ce[2], ce[3], ne[2], ne[3], s);
    }
    for (int m = 2; m < 4; ++m) {
      tmp = cl[m]; cl[m] = nl[m]; nl[m] = tmp;
      tmp = ce[m]; ce[m] = ne[m]; ne[m] = tmp;
    }
    for (int64_t s = 0; s < n_shots; ++s) {
      FN(adj_h)(&g, ones, cq, eta_hx, eta_hz, eta_ey, ce[0], ce[1], ne[0], ne[1], s);
      if (n_rec > 0 && grad_bg_r)
        FN(inject)(eta_ey, grad_bg_r + t * n_shots * n_rec, receivers_i, n_rec, N, s);
      if (n_src > 0 && grad_f0)
        FN(record)(grad_f0 + t * n_shots * n_src, eta_ey, sources_i, n_src, N, s);
      FN(adj_h)(&g, ca, cq, lam_hx, lam_hz, lam_ey, cl[0], cl[1], nl[0], nl[1], s);
      if (n_rec > 0 && grad_r)
        FN(inject)(lam_ey, grad_r + t * n_shots * n_rec, receivers_i, n_rec, N, s);
      if (n_src > 0 && grad_df)
        FN(record)(grad_df + t * n_shots * n_src, lam_ey, sources_i, n_src, N, s);
    }
    for (int m = 0; m < 2; ++m) {
      tmp = cl[m]; cl[m] = nl[m]; nl[m] = tmp;
      tmp = ce[m]; ce[m] = ne[m]; ne[m] = tmp;
    }
    ++swaps;
    if (t % step_ratio != 0) continue;
    const int64_t off = (t / step_ratio) * SN;
    FN(image_step)(&g, eta_ey, ey_store, off, bf16, kscale, grad_ca, ca_batched);
    FN(image_step)(&g, eta_ey, curl_store, off, bf16, kscale, grad_cb, cb_batched);
    FN(image_step)(&g, lam_ey, dey_store, off, bf16, kscale, grad_ca, ca_batched);
    FN(image_step)(&g, lam_ey, dcurl_store, off, bf16, kscale, grad_cb, cb_batched);
    FN(image_step)(&g, lam_ey, ey_store, off, bf16, kscale, grad_dca, ca_batched);
    FN(image_step)(&g, lam_ey, curl_store, off, bf16, kscale, grad_dcb, cb_batched);
  }
  if (swaps % 2 == 1)
    for (int m = 0; m < 4; ++m) {
      memcpy(m_lam[m], cl[m], (size_t)SN * sizeof(REAL));
      memcpy(m_eta[m], ce[m], (size_t)SN * sizeof(REAL));
    }
  free(ones);
  free(w);
}

#undef ORACLE_GEOM_INIT
#undef FN
#undef CAT2
#undef CAT2_
