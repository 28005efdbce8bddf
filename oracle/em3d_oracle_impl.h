/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle for the 3-D Maxwell (Yee) path.
 *
 * Included twice by em3d_oracle.c (REAL = float / double, SFX names the
 * instantiation).  Plain sequential C restating the reference's arithmetic
 * for stencil orders 2, 4, 6 and 8 (set by tide_oracle_em3d_set_stencil;
 * staggered differences and their transposes as
 * src/tide/csrc/common/staggered_grid.h:7-230, update domain
 * [FD_PAD, n - FD_PAD + 1) per axis with FD_PAD = order / 2):
 *
 *   forward H update        src/tide/csrc/em3d/maxwell_3d_inst.cpp:560-632
 *   forward E update        src/tide/csrc/em3d/maxwell_3d_inst.cpp:646-702
 *   E with snapshots        src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:755-868
 *   sources / receivers     src/tide/csrc/em3d/maxwell_3d_inst.cpp:300-348
 *   exact adjoint, E phase  src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:1478-1695
 *   exact adjoint, H phase  src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:1748-1829
 *   coefficient gradient    src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:2301-2368
 *   shot reduction          src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:2713-2727
 *   eps / sigma conversion  src/tide/csrc/em3d/maxwell_3d_inst.cpp:376-445
 *   reverse loop order      src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:4886-5190
 *
 * Compiled without FMA contraction and with IEEE division (d / kappa, as the
 * reference CPU backend and the reference's snapshot-storing CUDA kernel
 * do), so the float forward equals the reference CPU forward bit for bit.
 * CPML memories are full [S, nz, ny, nx] arrays here (the CUDA ABI passes
 * them compacted along their axis; tests convert).
 *
 * Field order: ex, ey, ez, hx, hy, hz.  Forward memories (reference ABI
 * order): m_hz_y, m_hy_z, m_hx_z, m_hz_x, m_hy_x, m_hx_y, m_ey_z, m_ez_y,
 * m_ez_x, m_ex_z, m_ex_y, m_ey_x.  Adjoint memories (reference ABI order):
 * ey_z, ez_y, ez_x, ex_z, ex_y, ey_x, hz_y, hy_z, hx_z, hz_x, hy_x, hx_y.
 * Profiles: az bz azh bzh ay by ayh byh ax bx axh bxh kz kzh ky kyh kx kxh.
 * Snapshots (device mode, [n_store, S, nz, ny, nx]): ex ey ez curl_x curl_y
 * curl_z; fmt 1 = bf16 (round to nearest even).
 */

#define CAT2_(a, b) a##_##b
#define CAT2(a, b) CAT2_(a, b)
#define FN(name) CAT2(name, SFX)

typedef struct {
  int64_t S, nz, ny, nx, N;
  REAL rdz, rdy, rdx;
  int64_t z0, y0, x0, z1, y1, x1;  /* integer-grid strips: c < c0 || c >= c1 */
  int64_t z1h, y1h, x1h;           /* half-grid strips:    c < c0 || c >= c1h */
  const REAL *p[18];
  int ca_b, cb_b, cq_b;
  int st, P;  /* stencil order, FD_PAD */
} FN(g3);

#ifndef EM3D_ORACLE_ENUMS
#define EM3D_ORACLE_ENUMS
enum { AZ, BZ, AZH, BZH, AY, BY, AYH, BYH, AX, BX, AXH, BXH, KZ, KZH, KY, KYH, KX, KXH };
/* Adjoint memories, ABI order. */
enum { L_EY_Z, L_EZ_Y, L_EZ_X, L_EX_Z, L_EX_Y, L_EY_X, L_HZ_Y, L_HY_Z, L_HX_Z, L_HZ_X, L_HY_X, L_HX_Y };
#endif

static inline int FN(active)(const FN(g3) * g, int64_t z, int64_t y, int64_t x) {
  const int64_t P = g->P;
  return z >= P && z < g->nz - P + 1 && y >= P && y < g->ny - P + 1 && x >= P &&
         x < g->nx - P + 1;
}
static inline int64_t FN(mi)(const FN(g3) * g, int64_t s, int64_t z, int64_t y, int64_t x) {
  return ((s * g->nz + z) * g->ny + y) * g->nx + x;
}

/* Staggered-grid coefficient m of an order-st difference. */
static inline REAL FN(cf)(int st, int m) {
  switch (st) {
    case 4: return m == 0 ? (REAL)(9.0 / 8.0) : (REAL)(-1.0 / 24.0);
    case 6: return m == 0 ? (REAL)(75.0 / 64.0) : m == 1 ? (REAL)(-25.0 / 384.0) : (REAL)(3.0 / 640.0);
    case 8:
      return m == 0 ? (REAL)(1225.0 / 1024.0)
             : m == 1 ? (REAL)(-245.0 / 3072.0)
             : m == 2 ? (REAL)(49.0 / 5120.0)
                      : (REAL)(-5.0 / 7168.0);
    default: return (REAL)1;
  }
}
/* Integer-grid difference (DIFF?1) of f at flat index i along stride sd. */
static inline REAL FN(d1)(const FN(g3) * g, const REAL *f, int64_t i, int64_t sd, REAL rd) {
  if (g->st == 2) return (f[i] - f[i - sd]) * rd;
  REAL acc = FN(cf)(g->st, 0) * (f[i] - f[i - sd]);
  for (int m = 1; m < g->P; ++m) acc = acc + FN(cf)(g->st, m) * (f[i + m * sd] - f[i - (m + 1) * sd]);
  return acc * rd;
}
/* Half-grid difference (DIFF?H1). */
static inline REAL FN(dh)(const FN(g3) * g, const REAL *f, int64_t i, int64_t sd, REAL rd) {
  if (g->st == 2) return (f[i + sd] - f[i]) * rd;
  REAL acc = FN(cf)(g->st, 0) * (f[i + sd] - f[i]);
  for (int m = 1; m < g->P; ++m) acc = acc + FN(cf)(g->st, m) * (f[i + (m + 1) * sd] - f[i - m * sd]);
  return acc * rd;
}
/* Transpose of a difference over raw terms (DIFF?1_ADJ(C, 1) and
 * DIFF?H1_ADJ(C, 1)): r[P - 1 - m] and r[P + m] are the raw terms paired by
 * coefficient m (offsets -m and m + 1 for the integer grid, -m - 1 and m for
 * the half grid; r holds offsets from -P + 1, resp. -P). */
static inline REAL FN(tadj)(const FN(g3) * g, const REAL *r, REAL rd) {
  const int P = g->P;
  if (g->st == 2) return (r[P - 1] * (REAL)1 - r[P] * (REAL)1) * rd;
  REAL acc = FN(cf)(g->st, 0) * (r[P - 1] * (REAL)1 - r[P] * (REAL)1);
  for (int m = 1; m < P; ++m)
    acc = acc + FN(cf)(g->st, m) * (r[P - 1 - m] * (REAL)1 - r[P + m] * (REAL)1);
  return acc * rd;
}

static void FN(step_h)(const FN(g3) * g, const REAL *cq, REAL **F, REAL **M) {
  REAL *ex = F[0], *ey = F[1], *ez = F[2], *hx = F[3], *hy = F[4], *hz = F[5];
  REAL *m_ey_z = M[6], *m_ez_y = M[7], *m_ez_x = M[8], *m_ex_z = M[9], *m_ex_y = M[10],
       *m_ey_x = M[11];
  const int64_t sz = g->ny * g->nx, sy = g->nx, P = g->P;
  for (int64_t s = 0; s < g->S; ++s)
    for (int64_t z = P; z < g->nz - P + 1; ++z)
      for (int64_t y = P; y < g->ny - P + 1; ++y)
        for (int64_t x = P; x < g->nx - P + 1; ++x) {
          const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
          const REAL c = cq[g->cq_b ? i : j];
          const int pz = z < g->z0 || z >= g->z1h, py = y < g->y0 || y >= g->y1h,
                    px = x < g->x0 || x >= g->x1h;
          REAL dEy_dz = 0, dEz_dy = 0, dEz_dx = 0, dEx_dz = 0, dEx_dy = 0, dEy_dx = 0;
          if (z < g->nz - P) {
            REAL d = FN(dh)(g, ey, i, sz, g->rdz);
            if (pz) {
              m_ey_z[i] = g->p[BZH][z] * m_ey_z[i] + g->p[AZH][z] * d;
              d = d / g->p[KZH][z] + m_ey_z[i];
            }
            dEy_dz = d;
          }
          if (y < g->ny - P) {
            REAL d = FN(dh)(g, ez, i, sy, g->rdy);
            if (py) {
              m_ez_y[i] = g->p[BYH][y] * m_ez_y[i] + g->p[AYH][y] * d;
              d = d / g->p[KYH][y] + m_ez_y[i];
            }
            dEz_dy = d;
          }
          if (x < g->nx - P) {
            REAL d = FN(dh)(g, ez, i, 1, g->rdx);
            if (px) {
              m_ez_x[i] = g->p[BXH][x] * m_ez_x[i] + g->p[AXH][x] * d;
              d = d / g->p[KXH][x] + m_ez_x[i];
            }
            dEz_dx = d;
          }
          if (z < g->nz - P) {
            REAL d = FN(dh)(g, ex, i, sz, g->rdz);
            if (pz) {
              m_ex_z[i] = g->p[BZH][z] * m_ex_z[i] + g->p[AZH][z] * d;
              d = d / g->p[KZH][z] + m_ex_z[i];
            }
            dEx_dz = d;
          }
          if (y < g->ny - P) {
            REAL d = FN(dh)(g, ex, i, sy, g->rdy);
            if (py) {
              m_ex_y[i] = g->p[BYH][y] * m_ex_y[i] + g->p[AYH][y] * d;
              d = d / g->p[KYH][y] + m_ex_y[i];
            }
            dEx_dy = d;
          }
          if (x < g->nx - P) {
            REAL d = FN(dh)(g, ey, i, 1, g->rdx);
            if (px) {
              m_ey_x[i] = g->p[BXH][x] * m_ey_x[i] + g->p[AXH][x] * d;
              d = d / g->p[KXH][x] + m_ey_x[i];
            }
            dEy_dx = d;
          }
          hx[i] = hx[i] - c * (dEy_dz - dEz_dy);
          hy[i] = hy[i] - c * (dEz_dx - dEx_dz);
          hz[i] = hz[i] - c * (dEx_dy - dEy_dx);
        }
}

static inline uint16_t FN(bf16)(REAL v) {
  float f = (float)v;
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) return (uint16_t)((u >> 16) | 0x40);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
static inline REAL FN(unbf16)(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  memcpy(&f, &u, 4);
  return (REAL)f;
}
static inline void FN(put)(void *st, int fmt, int64_t i, REAL v) {
  if (fmt) ((uint16_t *)st)[i] = FN(bf16)(v);
  else ((REAL *)st)[i] = v;
}
static inline REAL FN(get)(const void *st, int fmt, int64_t i) {
  return fmt ? FN(unbf16)(((const uint16_t *)st)[i]) : ((const REAL *)st)[i];
}

/* E update; st[6] (ex, ey, ez, curl x/y/z snapshots of this step) or NULLs. */
static void FN(step_e)(const FN(g3) * g, const REAL *ca, const REAL *cb, REAL **F, REAL **M,
                       void **st, int fmt) {
  REAL *ex = F[0], *ey = F[1], *ez = F[2], *hx = F[3], *hy = F[4], *hz = F[5];
  REAL *m_hz_y = M[0], *m_hy_z = M[1], *m_hx_z = M[2], *m_hz_x = M[3], *m_hy_x = M[4],
       *m_hx_y = M[5];
  const int64_t sz = g->ny * g->nx, sy = g->nx, P = g->P;
  for (int64_t s = 0; s < g->S; ++s)
    for (int64_t z = P; z < g->nz - P + 1; ++z)
      for (int64_t y = P; y < g->ny - P + 1; ++y)
        for (int64_t x = P; x < g->nx - P + 1; ++x) {
          const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
          const REAL a = ca[g->ca_b ? i : j], b = cb[g->cb_b ? i : j];
          REAL dHy_dz = FN(d1)(g, hy, i, sz, g->rdz);
          REAL dHz_dy = FN(d1)(g, hz, i, sy, g->rdy);
          REAL dHz_dx = FN(d1)(g, hz, i, 1, g->rdx);
          REAL dHx_dz = FN(d1)(g, hx, i, sz, g->rdz);
          REAL dHx_dy = FN(d1)(g, hx, i, sy, g->rdy);
          REAL dHy_dx = FN(d1)(g, hy, i, 1, g->rdx);
          if (z < g->z0 || z >= g->z1) {
            m_hy_z[i] = g->p[BZ][z] * m_hy_z[i] + g->p[AZ][z] * dHy_dz;
            dHy_dz = dHy_dz / g->p[KZ][z] + m_hy_z[i];
            m_hx_z[i] = g->p[BZ][z] * m_hx_z[i] + g->p[AZ][z] * dHx_dz;
            dHx_dz = dHx_dz / g->p[KZ][z] + m_hx_z[i];
          }
          if (y < g->y0 || y >= g->y1) {
            m_hz_y[i] = g->p[BY][y] * m_hz_y[i] + g->p[AY][y] * dHz_dy;
            dHz_dy = dHz_dy / g->p[KY][y] + m_hz_y[i];
            m_hx_y[i] = g->p[BY][y] * m_hx_y[i] + g->p[AY][y] * dHx_dy;
            dHx_dy = dHx_dy / g->p[KY][y] + m_hx_y[i];
          }
          if (x < g->x0 || x >= g->x1) {
            m_hz_x[i] = g->p[BX][x] * m_hz_x[i] + g->p[AX][x] * dHz_dx;
            dHz_dx = dHz_dx / g->p[KX][x] + m_hz_x[i];
            m_hy_x[i] = g->p[BX][x] * m_hy_x[i] + g->p[AX][x] * dHy_dx;
            dHy_dx = dHy_dx / g->p[KX][x] + m_hy_x[i];
          }
          const REAL cx = dHy_dz - dHz_dy, cy = dHz_dx - dHx_dz, cz = dHx_dy - dHy_dx;
          if (st && st[0]) {
            FN(put)(st[0], fmt, i, ex[i]);
            FN(put)(st[1], fmt, i, ey[i]);
            FN(put)(st[2], fmt, i, ez[i]);
          }
          if (st && st[3]) {
            FN(put)(st[3], fmt, i, cx);
            FN(put)(st[4], fmt, i, cy);
            FN(put)(st[5], fmt, i, cz);
          }
          ex[i] = a * ex[i] + b * cx;
          ey[i] = a * ey[i] + b * cy;
          ez[i] = a * ez[i] + b * cz;
        }
}

/* Born E half-step (maxwell_3d_inst.cpp:1390-1475): background and scattered
 * curls with their own CPML memories; the scattered update adds
 * dca E^n + dcb curl H^n of the background. */
static void FN(step_e_born)(const FN(g3) * g, const REAL *ca, const REAL *cb, const REAL *dca,
                            const REAL *dcb, REAL **F, REAL **M, REAL **DF, REAL **DM,
                            void **st, int fmt) {
  const int64_t sz = g->ny * g->nx, sy = g->nx, P = g->P;
  for (int64_t s = 0; s < g->S; ++s)
    for (int64_t z = P; z < g->nz - P + 1; ++z)
      for (int64_t y = P; y < g->ny - P + 1; ++y)
        for (int64_t x = P; x < g->nx - P + 1; ++x) {
          const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
          const REAL a = ca[g->ca_b ? i : j], b = cb[g->cb_b ? i : j];
          const REAL da = dca[g->ca_b ? i : j], db = dcb[g->cb_b ? i : j];
          const int pz = z < g->z0 || z >= g->z1, py = y < g->y0 || y >= g->y1,
                    px = x < g->x0 || x >= g->x1;
          REAL c[2][3];
          for (int w = 0; w < 2; ++w) {
            REAL **H = w ? DF : F, **Q = w ? DM : M;
            const REAL *hx = H[3], *hy = H[4], *hz = H[5];
            REAL dHy_dz = FN(d1)(g, hy, i, sz, g->rdz);
            REAL dHz_dy = FN(d1)(g, hz, i, sy, g->rdy);
            REAL dHz_dx = FN(d1)(g, hz, i, 1, g->rdx);
            REAL dHx_dz = FN(d1)(g, hx, i, sz, g->rdz);
            REAL dHx_dy = FN(d1)(g, hx, i, sy, g->rdy);
            REAL dHy_dx = FN(d1)(g, hy, i, 1, g->rdx);
            if (pz) {
              Q[1][i] = g->p[BZ][z] * Q[1][i] + g->p[AZ][z] * dHy_dz;
              dHy_dz = dHy_dz / g->p[KZ][z] + Q[1][i];
              Q[2][i] = g->p[BZ][z] * Q[2][i] + g->p[AZ][z] * dHx_dz;
              dHx_dz = dHx_dz / g->p[KZ][z] + Q[2][i];
            }
            if (py) {
              Q[0][i] = g->p[BY][y] * Q[0][i] + g->p[AY][y] * dHz_dy;
              dHz_dy = dHz_dy / g->p[KY][y] + Q[0][i];
              Q[5][i] = g->p[BY][y] * Q[5][i] + g->p[AY][y] * dHx_dy;
              dHx_dy = dHx_dy / g->p[KY][y] + Q[5][i];
            }
            if (px) {
              Q[3][i] = g->p[BX][x] * Q[3][i] + g->p[AX][x] * dHz_dx;
              dHz_dx = dHz_dx / g->p[KX][x] + Q[3][i];
              Q[4][i] = g->p[BX][x] * Q[4][i] + g->p[AX][x] * dHy_dx;
              dHy_dx = dHy_dx / g->p[KX][x] + Q[4][i];
            }
            c[w][0] = dHy_dz - dHz_dy;
            c[w][1] = dHz_dx - dHx_dz;
            c[w][2] = dHx_dy - dHy_dx;
          }
          /* snapshots before the update (maxwell_3d_cuda_inst.cu:1291-1340):
           * background E^n, curl H^n, scattered E^n, scattered curl */
          for (int k = 0; k < 3; ++k) {
            if (st && st[k]) FN(put)(st[k], fmt, i, F[k][i]);
            if (st && st[3 + k]) FN(put)(st[3 + k], fmt, i, c[0][k]);
            if (st && st[6 + k]) FN(put)(st[6 + k], fmt, i, DF[k][i]);
            if (st && st[9 + k]) FN(put)(st[9 + k], fmt, i, c[1][k]);
          }
          for (int k = 0; k < 3; ++k) {
            const REAL e_old = F[k][i];
            DF[k][i] = a * DF[k][i] + b * c[1][k] + da * e_old + db * c[0][k];
            F[k][i] = a * e_old + b * c[0][k];
          }
        }
}

static void FN(inject)(REAL *field, const REAL *vals, const int64_t *idx, int64_t S, int64_t n,
                       int64_t N) {
  for (int64_t s = 0; s < S; ++s)
    for (int64_t k = 0; k < n; ++k) {
      const int64_t c = idx[s * n + k];
      if (c >= 0) field[s * N + c] = field[s * N + c] + vals[s * n + k];
    }
}
static void FN(record)(REAL *out, const REAL *field, const int64_t *idx, int64_t S, int64_t n,
                       int64_t N) {
  for (int64_t s = 0; s < S; ++s)
    for (int64_t k = 0; k < n; ++k) {
      const int64_t c = idx[s * n + k];
      out[s * n + k] = c >= 0 ? field[s * N + c] : (REAL)0;
    }
}

static void FN(setup)(FN(g3) * g, const REAL **prof, REAL rdz, REAL rdy, REAL rdx, int64_t S,
                      int64_t nz, int64_t ny, int64_t nx, const int64_t *pml, int ca_b, int cb_b,
                      int cq_b) {
  g->S = S;
  g->nz = nz;
  g->ny = ny;
  g->nx = nx;
  g->N = nz * ny * nx;
  g->rdz = rdz;
  g->rdy = rdy;
  g->rdx = rdx;
  g->z0 = pml[0];
  g->y0 = pml[1];
  g->x0 = pml[2];
  g->z1 = pml[3];
  g->y1 = pml[4];
  g->x1 = pml[5];
  g->z1h = g->z1 > g->z0 ? g->z1 - 1 : g->z0;
  g->y1h = g->y1 > g->y0 ? g->y1 - 1 : g->y0;
  g->x1h = g->x1 > g->x0 ? g->x1 - 1 : g->x0;
  for (int k = 0; k < 18; ++k) g->p[k] = prof[k];
  g->ca_b = ca_b;
  g->cb_b = cb_b;
  g->cq_b = cq_b;
  g->st = g_em3d_stencil;
  g->P = g_em3d_stencil / 2;
}

/* Forward over steps [start_t, start_t + nt).  store: 6 snapshot histories
 * (or NULLs), written at steps t % k == 0 into slot t / k. */
void FN(tide_oracle_em3d_forward)(const REAL *ca, const REAL *cb, const REAL *cq, const REAL *f,
                                  REAL **F, REAL **M, REAL *r, const REAL **prof,
                                  const int64_t *src_i, const int64_t *rec_i, REAL rdz, REAL rdy,
                                  REAL rdx, int64_t nt, int64_t S, int64_t nz, int64_t ny,
                                  int64_t nx, int64_t n_src, int64_t n_rec, int64_t start_t,
                                  const int64_t *pml, int ca_b, int cb_b, int cq_b, int src_comp,
                                  int rec_comp, void **store, int64_t k, int fmt) {
  FN(g3) g;
  FN(setup)(&g, prof, rdz, rdy, rdx, S, nz, ny, nx, pml, ca_b, cb_b, cq_b);
  const size_t esz = fmt ? 2 : sizeof(REAL);
  for (int64_t t = start_t; t < start_t + nt; ++t) {
    FN(step_h)(&g, cq, F, M);
    void *st[6] = {0, 0, 0, 0, 0, 0};
    if (store && k > 0 && t % k == 0)
      for (int c = 0; c < 6; ++c)
        if (store[c]) st[c] = (char *)store[c] + (size_t)(t / k) * (size_t)(S * g.N) * esz;
    FN(step_e)(&g, ca, cb, F, M, store ? st : 0, fmt);
    if (n_src > 0 && f && src_i) FN(inject)(F[src_comp], f + t * S * n_src, src_i, S, n_src, g.N);
    if (n_rec > 0 && r && rec_i) FN(record)(r + t * S * n_rec, F[rec_comp], rec_i, S, n_rec, g.N);
  }
}

/* Born forward over steps [start_t, start_t + nt) (maxwell_3d_inst.cpp:
 * 1100-1527): F/M background, DF/DM scattered state; r records the scattered
 * and bg_r (may be NULL) the background receiver component.  store: 12
 * snapshot histories (background E, curl H, scattered E, scattered curl; any
 * may be NULL) written at steps t % k == 0 into slot t / k, or NULL. */
void FN(tide_oracle_em3d_born_forward_store)(
    const REAL *ca, const REAL *cb, const REAL *cq, const REAL *dca, const REAL *dcb,
    const REAL *f0, const REAL *df, REAL **F, REAL **M, REAL **DF, REAL **DM, REAL *r,
    REAL *bg_r, const REAL **prof, const int64_t *src_i, const int64_t *rec_i, REAL rdz,
    REAL rdy, REAL rdx, int64_t nt, int64_t S, int64_t nz, int64_t ny, int64_t nx,
    int64_t n_src, int64_t n_rec, int64_t start_t, const int64_t *pml, int ca_b, int cb_b,
    int cq_b, int src_comp, int rec_comp, void **store, int64_t k, int fmt) {
  FN(g3) g;
  FN(setup)(&g, prof, rdz, rdy, rdx, S, nz, ny, nx, pml, ca_b, cb_b, cq_b);
  const size_t esz = fmt ? 2 : sizeof(REAL);
  for (int64_t t = start_t; t < start_t + nt; ++t) {
    FN(step_h)(&g, cq, F, M);
    FN(step_h)(&g, cq, DF, DM);
    void *st[12] = {0};
    if (store && k > 0 && t % k == 0)
      for (int c = 0; c < 12; ++c)
        if (store[c]) st[c] = (char *)store[c] + (size_t)(t / k) * (size_t)(S * g.N) * esz;
    FN(step_e_born)(&g, ca, cb, dca, dcb, F, M, DF, DM, store ? st : 0, fmt);
    if (n_src > 0 && f0 && src_i) {
      FN(inject)(F[src_comp], f0 + t * S * n_src, src_i, S, n_src, g.N);
      FN(inject)(DF[src_comp], df + t * S * n_src, src_i, S, n_src, g.N);
    }
    if (n_rec > 0 && r && rec_i) FN(record)(r + t * S * n_rec, DF[rec_comp], rec_i, S, n_rec, g.N);
    if (n_rec > 0 && bg_r && rec_i)
      FN(record)(bg_r + t * S * n_rec, F[rec_comp], rec_i, S, n_rec, g.N);
  }
}

void FN(tide_oracle_em3d_born_forward)(const REAL *ca, const REAL *cb, const REAL *cq,
                                       const REAL *dca, const REAL *dcb, const REAL *f0,
                                       const REAL *df, REAL **F, REAL **M, REAL **DF, REAL **DM,
                                       REAL *r, REAL *bg_r, const REAL **prof,
                                       const int64_t *src_i, const int64_t *rec_i, REAL rdz,
                                       REAL rdy, REAL rdx, int64_t nt, int64_t S, int64_t nz,
                                       int64_t ny, int64_t nx, int64_t n_src, int64_t n_rec,
                                       int64_t start_t, const int64_t *pml, int ca_b, int cb_b,
                                       int cq_b, int src_comp, int rec_comp) {
  FN(tide_oracle_em3d_born_forward_store)(ca, cb, cq, dca, dcb, f0, df, F, M, DF, DM, r, bg_r,
                                          prof, src_i, rec_i, rdz, rdy, rdx, nt, S, nz, ny, nx,
                                          n_src, n_rec, start_t, pml, ca_b, cb_b, cq_b, src_comp,
                                          rec_comp, 0, 0, 0);
}

/* Raw adjoint terms at the offset cell o (reference raw_e_side / raw_h_side). */
static inline REAL FN(raw_e)(const FN(g3) * g, const REAL *coef, int cb_batched, const REAL *lam,
                             const REAL *mem, int axis, int neg, int64_t s, int64_t z, int64_t y,
                             int64_t x) {
  if (!FN(active)(g, z, y, x)) return 0;
  const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
  REAL q = coef[cb_batched ? i : j] * lam[i];
  if (neg) q = -q;
  const int64_t c = axis == 0 ? z : axis == 1 ? y : x;
  const int64_t lo = axis == 0 ? g->z0 : axis == 1 ? g->y0 : g->x0;
  const int64_t hi = axis == 0 ? g->z1 : axis == 1 ? g->y1 : g->x1;
  const REAL *A = g->p[axis == 0 ? AZ : axis == 1 ? AY : AX];
  const REAL *B = g->p[axis == 0 ? BZ : axis == 1 ? BY : BX];
  const REAL *K = g->p[axis == 0 ? KZ : axis == 1 ? KY : KX];
  const REAL m_used = B[c] * mem[i] + q;
  return (c < lo || c >= hi) ? (A[c] * m_used + q / K[c]) : q;
}
static inline REAL FN(raw_h)(const FN(g3) * g, const REAL *coef, int cq_batched, const REAL *lam,
                             const REAL *mem, int axis, int neg, int64_t s, int64_t z, int64_t y,
                             int64_t x) {
  if (!FN(active)(g, z, y, x)) return 0;
  const int64_t c = axis == 0 ? z : axis == 1 ? y : x;
  const int64_t n = axis == 0 ? g->nz : axis == 1 ? g->ny : g->nx;
  if (c >= n - g->P) return 0;
  const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
  REAL q = coef[cq_batched ? i : j] * lam[i];
  if (neg) q = -q;
  const int64_t lo = axis == 0 ? g->z0 : axis == 1 ? g->y0 : g->x0;
  const int64_t hi = axis == 0 ? g->z1h : axis == 1 ? g->y1h : g->x1h;
  const REAL *A = g->p[axis == 0 ? AZH : axis == 1 ? AYH : AXH];
  const REAL *B = g->p[axis == 0 ? BZH : axis == 1 ? BYH : BXH];
  const REAL *K = g->p[axis == 0 ? KZH : axis == 1 ? KYH : KXH];
  const REAL m_used = B[c] * mem[i] + q;
  return (c < lo || c >= hi) ? (A[c] * m_used + q / K[c]) : q;
}

static void FN(adj_e)(const FN(g3) * g, const REAL *cb, REAL **L, REAL **cur, REAL **nxt) {
  REAL *lex = L[0], *ley = L[1], *lez = L[2], *lhx = L[3], *lhy = L[4], *lhz = L[5];
  const int64_t P = g->P;
  for (int64_t s = 0; s < g->S; ++s)
    for (int64_t z = P; z < g->nz - P + 1; ++z)
      for (int64_t y = P; y < g->ny - P + 1; ++y)
        for (int64_t x = P; x < g->nx - P + 1; ++x) {
          const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
          const REAL c = cb[g->cb_b ? i : j];
          const REAL qx = c * lex[i], qy = c * ley[i], qz = c * lez[i];
          const int pz = z < g->z0 || z >= g->z1, py = y < g->y0 || y >= g->y1,
                    px = x < g->x0 || x >= g->x1;
          nxt[L_HY_Z][i] = pz ? g->p[BZ][z] * cur[L_HY_Z][i] + qx : (REAL)0;
          nxt[L_HX_Z][i] = pz ? g->p[BZ][z] * cur[L_HX_Z][i] - qy : (REAL)0;
          nxt[L_HZ_Y][i] = py ? g->p[BY][y] * cur[L_HZ_Y][i] - qx : (REAL)0;
          nxt[L_HX_Y][i] = py ? g->p[BY][y] * cur[L_HX_Y][i] + qz : (REAL)0;
          nxt[L_HZ_X][i] = px ? g->p[BX][x] * cur[L_HZ_X][i] + qy : (REAL)0;
          nxt[L_HY_X][i] = px ? g->p[BX][x] * cur[L_HY_X][i] - qz : (REAL)0;
          const int cb_b = g->cb_b;
          /* raw terms at offsets -P+1 .. P along one axis (DIFF?1_ADJ) */
#define RE(dst, lam, mem, ax, ng)                                                         \
  for (int o = 1 - (int)P; o <= (int)P; ++o)                                                \
    dst[o + P - 1] = FN(raw_e)(g, cb, cb_b, lam, cur[mem], ax, ng, s, z + (ax == 0 ? o : 0), \
                               y + (ax == 1 ? o : 0), x + (ax == 2 ? o : 0));
          REAL r1[8], r2[8];
          RE(r1, ley, L_HX_Z, 0, 1)
          RE(r2, lez, L_HX_Y, 1, 0)
          lhx[i] = lhx[i] + (FN(tadj)(g, r1, g->rdz) + FN(tadj)(g, r2, g->rdy));
          RE(r1, lex, L_HY_Z, 0, 0)
          RE(r2, lez, L_HY_X, 2, 1)
          lhy[i] = lhy[i] + (FN(tadj)(g, r1, g->rdz) + FN(tadj)(g, r2, g->rdx));
          RE(r1, lex, L_HZ_Y, 1, 1)
          RE(r2, ley, L_HZ_X, 2, 0)
          lhz[i] = lhz[i] + (FN(tadj)(g, r1, g->rdy) + FN(tadj)(g, r2, g->rdx));
#undef RE
        }
}

static void FN(adj_h)(const FN(g3) * g, const REAL *ca, const REAL *cq, REAL **L, REAL **cur,
                      REAL **nxt) {
  REAL *lex = L[0], *ley = L[1], *lez = L[2], *lhx = L[3], *lhy = L[4], *lhz = L[5];
  const int64_t P = g->P;
  for (int64_t s = 0; s < g->S; ++s)
    for (int64_t z = P; z < g->nz - P + 1; ++z)
      for (int64_t y = P; y < g->ny - P + 1; ++y)
        for (int64_t x = P; x < g->nx - P + 1; ++x) {
          const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
          const REAL c = cq[g->cq_b ? i : j];
          const int pz = z < g->nz - P && (z < g->z0 || z >= g->z1h);
          const int py = y < g->ny - P && (y < g->y0 || y >= g->y1h);
          const int px = x < g->nx - P && (x < g->x0 || x >= g->x1h);
          nxt[L_EY_Z][i] = pz ? g->p[BZH][z] * cur[L_EY_Z][i] - c * lhx[i] : (REAL)0;
          nxt[L_EX_Z][i] = pz ? g->p[BZH][z] * cur[L_EX_Z][i] + c * lhy[i] : (REAL)0;
          nxt[L_EZ_Y][i] = py ? g->p[BYH][y] * cur[L_EZ_Y][i] + c * lhx[i] : (REAL)0;
          nxt[L_EX_Y][i] = py ? g->p[BYH][y] * cur[L_EX_Y][i] - c * lhz[i] : (REAL)0;
          nxt[L_EZ_X][i] = px ? g->p[BXH][x] * cur[L_EZ_X][i] - c * lhy[i] : (REAL)0;
          nxt[L_EY_X][i] = px ? g->p[BXH][x] * cur[L_EY_X][i] + c * lhz[i] : (REAL)0;
          const REAL a = ca[g->ca_b ? i : j];
          lex[i] = a * lex[i];
          ley[i] = a * ley[i];
          lez[i] = a * lez[i];
          const int cq_b = g->cq_b;
          /* raw terms at offsets -P .. P-1 along one axis (DIFF?H1_ADJ) */
#define RH(dst, lam, mem, ax, ng)                                                         \
  for (int o = -(int)P; o < (int)P; ++o)                                                    \
    dst[o + P] = FN(raw_h)(g, cq, cq_b, lam, cur[mem], ax, ng, s, z + (ax == 0 ? o : 0),     \
                           y + (ax == 1 ? o : 0), x + (ax == 2 ? o : 0));
          REAL r1[8], r2[8];
          RH(r1, lhx, L_EY_Z, 0, 1)
          RH(r2, lhz, L_EY_X, 2, 0)
          ley[i] = ley[i] + (FN(tadj)(g, r1, g->rdz) + FN(tadj)(g, r2, g->rdx));
          RH(r1, lhy, L_EX_Z, 0, 0)
          RH(r2, lhz, L_EX_Y, 1, 1)
          lex[i] = lex[i] + (FN(tadj)(g, r1, g->rdz) + FN(tadj)(g, r2, g->rdy));
          RH(r1, lhx, L_EZ_Y, 1, 0)
          RH(r2, lhy, L_EZ_X, 2, 1)
          lez[i] = lez[i] + (FN(tadj)(g, r1, g->rdy) + FN(tadj)(g, r2, g->rdx));
#undef RH
        }
}

/* Exact adjoint over t = start_t-1 down to start_t-nt.  lmem: the 12 adjoint
 * memories (updated in place, ping-pong with internal buffers).  Gradients
 * accumulate: grad_ca / grad_cb model-shaped (per shot when batched); with
 * several unbatched shots per-shot sums are kept and added once at the end,
 * in shot order, as the reference does.  grad_eps / grad_sigma (optional)
 * receive the conversion of the final grad_ca / grad_cb. */
void FN(tide_oracle_em3d_backward)(const REAL *ca, const REAL *cb, const REAL *cq,
                                   const REAL *grad_r, REAL **L, REAL **lmem, void **store,
                                   REAL *grad_f, REAL *grad_ca, REAL *grad_cb, REAL *grad_eps,
                                   REAL *grad_sigma, REAL dt, const REAL **prof,
                                   const int64_t *src_i, const int64_t *rec_i, REAL rdz, REAL rdy,
                                   REAL rdx, int64_t nt, int64_t S, int64_t nz, int64_t ny,
                                   int64_t nx, int64_t n_src, int64_t n_rec, int64_t k, int fmt,
                                   int64_t start_t, const int64_t *pml, int ca_b, int cb_b,
                                   int cq_b, int src_comp, int rec_comp, int need_ca,
                                   int need_cb) {
  FN(g3) g;
  FN(setup)(&g, prof, rdz, rdy, rdx, S, nz, ny, nx, pml, ca_b, cb_b, cq_b);
  const int64_t tot = S * g.N;
  REAL *scratch = (REAL *)calloc((size_t)(12 * tot), sizeof(REAL));
  REAL *cur[12], *nxt[12];
  for (int m = 0; m < 12; ++m) {
    cur[m] = lmem[m];
    nxt[m] = scratch + m * tot;
  }
  const int shot_ca = need_ca && !ca_b && S > 1, shot_cb = need_cb && !cb_b && S > 1;
  REAL *gca_s = shot_ca ? (REAL *)calloc((size_t)tot, sizeof(REAL)) : 0;
  REAL *gcb_s = shot_cb ? (REAL *)calloc((size_t)tot, sizeof(REAL)) : 0;
  const size_t esz = fmt ? 2 : sizeof(REAL);
  for (int64_t t = start_t - 1; t >= start_t - nt; --t) {
    FN(adj_e)(&g, cb, L, cur, nxt);
    /* H phase reads the H-phase memories of the current step */
    FN(adj_h)(&g, ca, cq, L, cur, nxt);
    if (n_rec > 0 && grad_r && rec_i) FN(inject)(L[rec_comp], grad_r + t * S * n_rec, rec_i, S, n_rec, g.N);
    if (n_src > 0 && grad_f && src_i) FN(record)(grad_f + t * S * n_src, L[src_comp], src_i, S, n_src, g.N);
    if (k > 0 && t % k == 0 && store) {
      const size_t off = (size_t)(t / k) * (size_t)tot * esz;
      for (int64_t s = 0; s < S; ++s)
        for (int64_t z = g.P; z < nz - g.P + 1; ++z)
          for (int64_t y = g.P; y < ny - g.P + 1; ++y)
            for (int64_t x = g.P; x < nx - g.P + 1; ++x) {
              const int64_t i = FN(mi)(&g, s, z, y, x), j = i - s * g.N;
              const REAL lx = L[0][i], ly = L[1][i], lz = L[2][i];
              if (need_ca && store[0]) {
                const char *b0 = (const char *)store[0] + off, *b1 = (const char *)store[1] + off,
                           *b2 = (const char *)store[2] + off;
                const REAL acc = lx * FN(get)(b0, fmt, i) + ly * FN(get)(b1, fmt, i) +
                                 lz * FN(get)(b2, fmt, i);
                const REAL sc = acc * (REAL)k;
                if (ca_b) grad_ca[i] = grad_ca[i] + sc;
                else if (S == 1) grad_ca[j] = grad_ca[j] + sc;
                else gca_s[i] = gca_s[i] + sc;
              }
              if (need_cb && store[3]) {
                const char *b0 = (const char *)store[3] + off, *b1 = (const char *)store[4] + off,
                           *b2 = (const char *)store[5] + off;
                const REAL acc = lx * FN(get)(b0, fmt, i) + ly * FN(get)(b1, fmt, i) +
                                 lz * FN(get)(b2, fmt, i);
                const REAL sc = acc * (REAL)k;
                if (cb_b) grad_cb[i] = grad_cb[i] + sc;
                else if (S == 1) grad_cb[j] = grad_cb[j] + sc;
                else gcb_s[i] = gcb_s[i] + sc;
              }
            }
    }
    for (int m = 0; m < 12; ++m) {
      REAL *tmp = cur[m];
      cur[m] = nxt[m];
      nxt[m] = tmp;
    }
  }
  for (int m = 0; m < 12; ++m)
    if (cur[m] != lmem[m]) memcpy(lmem[m], cur[m], (size_t)tot * sizeof(REAL));
  for (int w = 0; w < 2; ++w) {
    REAL *acc = w ? gcb_s : gca_s, *out = w ? grad_cb : grad_ca;
    if (!acc) continue;
    for (int64_t j = 0; j < g.N; ++j) {
      REAL sum = 0;
      for (int64_t s = 0; s < S; ++s) sum = sum + acc[s * g.N + j];
      out[j] = out[j] + sum;
    }
  }
  if (grad_eps || grad_sigma) {
    const REAL inv_dt = (REAL)1 / dt, ep0 = (REAL)8.8541878128e-12;
    const int64_t n = ca_b ? tot : g.N;
    for (int64_t o = 0; o < n; ++o) {
      const int64_t s = ca_b ? o / g.N : 0, j = o - s * g.N;
      const REAL av = ca[ca_b ? o : j], bv = cb[cb_b ? s * g.N + j : j], bsq = bv * bv;
      const REAL ga = need_ca && grad_ca ? grad_ca[o] : (REAL)0;
      const REAL gb = need_cb && grad_cb ? grad_cb[o] : (REAL)0;
      const REAL dca_de = ((REAL)1 - av) * bv * inv_dt, dcb_de = -bsq * inv_dt;
      const REAL dca_ds = -((REAL)0.5) * ((REAL)1 + av) * bv, dcb_ds = -((REAL)0.5) * bsq;
      if (grad_eps) grad_eps[o] = (ga * dca_de + gb * dcb_de) * ep0;
      if (grad_sigma) grad_sigma[o] = ga * dca_ds + gb * dcb_ds;
    }
  }
  free(scratch);
  free(gca_s);
  free(gcb_s);
}

/* One stored step's coefficient-gradient term of the fields F[0..2] against
 * the three snapshot histories st[0..2] (slot byte offset off), into grad
 * (batched), grad[j] (one shot) or the per-shot buffer shot (several shots). */
static void FN(image3)(const FN(g3) * g, REAL *const F[3], void *const st[3], size_t off,
                       int fmt, REAL kscale, REAL *grad, REAL *shot, int batched) {
  for (int64_t s = 0; s < g->S; ++s)
    for (int64_t z = g->P; z < g->nz - g->P + 1; ++z)
      for (int64_t y = g->P; y < g->ny - g->P + 1; ++y)
        for (int64_t x = g->P; x < g->nx - g->P + 1; ++x) {
          const int64_t i = FN(mi)(g, s, z, y, x), j = i - s * g->N;
          const REAL acc = F[0][i] * FN(get)((const char *)st[0] + off, fmt, i) +
                           F[1][i] * FN(get)((const char *)st[1] + off, fmt, i) +
                           F[2][i] * FN(get)((const char *)st[2] + off, fmt, i);
          const REAL sc = acc * kscale;
          if (batched) grad[i] = grad[i] + sc;
          else if (g->S == 1) grad[j] = grad[j] + sc;
          else shot[i] = shot[i] + sc;
        }
}

/* Second-order Born adjoint, 3-D (the reference's born_backward_bggrad,
 * maxwell_3d_cuda_inst.cu:5262-5900, in the formulation of the TM2D oracle):
 * lam (L, 6 fields + 12 memories) is the scattered state's adjoint driven by
 * grad_r, eta (E) the background's, driven by the scattered update's
 * dependence on the background: per step W = cb eta_E + dcb lam_E and
 * eta_E <- ca eta_E + dca lam_E on the update domain, the adjoint phases of
 * lam (cb, ca) and of eta (W for the E-phase input, unit ca), receivers
 * grad_r -> lam, sources grad_df <- lam and grad_f0 <- eta, then at stored
 * steps grad_ca += eta.E + lam.dE, grad_cb += eta.curl + lam.dcurl,
 * grad_dca += lam.E, grad_dcb += lam.curl (times k; per-shot buffers summed
 * over shots at the end).  store: background E x3, curl x3; dstore: the
 * scattered ones; full-layout memories. */
void FN(tide_oracle_em3d_born_bggrad)(
    const REAL *ca, const REAL *cb, const REAL *cq, const REAL *dca, const REAL *dcb,
    const REAL *grad_r, REAL **L, REAL **lmem, REAL **E, REAL **emem, void **store,
    void **dstore, REAL *grad_f0, REAL *grad_df, REAL *grad_ca, REAL *grad_cb, REAL *grad_dca,
    REAL *grad_dcb, const REAL **prof, const int64_t *src_i, const int64_t *rec_i, REAL rdz,
    REAL rdy, REAL rdx, int64_t nt, int64_t S, int64_t nz, int64_t ny, int64_t nx, int64_t n_src,
    int64_t n_rec, int64_t k, int fmt, int64_t start_t, const int64_t *pml, int ca_b, int cb_b,
    int cq_b, int src_comp, int rec_comp) {
  FN(g3) g;
  FN(setup)(&g, prof, rdz, rdy, rdx, S, nz, ny, nx, pml, ca_b, cb_b, cq_b);
  const int64_t tot = S * g.N;
  REAL *scratch = (REAL *)calloc((size_t)(24 * tot), sizeof(REAL));
  REAL *ones = (REAL *)malloc((size_t)tot * sizeof(REAL));
  REAL *w = (REAL *)calloc((size_t)(3 * tot), sizeof(REAL));
  for (int64_t i = 0; i < tot; ++i) ones[i] = (REAL)1;
  REAL *lc[12], *ln[12], *ec[12], *en[12];
  for (int m = 0; m < 12; ++m) {
    lc[m] = lmem[m];
    ln[m] = scratch + m * tot;
    ec[m] = emem[m];
    en[m] = scratch + (12 + m) * tot;
  }
  REAL *WE[6] = {w, w + tot, w + 2 * tot, E[3], E[4], E[5]};
  const int sh_a = !ca_b && S > 1, sh_b = !cb_b && S > 1;
  REAL *shot[4];
  for (int q = 0; q < 4; ++q)
    shot[q] = ((q % 2 == 0) ? sh_a : sh_b) ? (REAL *)calloc((size_t)tot, sizeof(REAL)) : 0;
  const size_t esz = fmt ? 2 : sizeof(REAL);
  for (int64_t t = start_t - 1; t >= start_t - nt; --t) {
    for (int64_t s = 0; s < S; ++s)
      for (int64_t z = g.P; z < nz - g.P + 1; ++z)
        for (int64_t y = g.P; y < ny - g.P + 1; ++y)
          for (int64_t x = g.P; x < nx - g.P + 1; ++x) {
            const int64_t i = FN(mi)(&g, s, z, y, x), j = i - s * g.N;
            const REAL a = ca[ca_b ? i : j], da = dca[ca_b ? i : j];
            const REAL b = cb[cb_b ? i : j], db = dcb[cb_b ? i : j];
            for (int c = 0; c < 3; ++c) {
              WE[c][i] = b * E[c][i] + db * L[c][i];
              E[c][i] = a * E[c][i] + da * L[c][i];
            }
          }
    FN(adj_e)(&g, cb, L, lc, ln);
    FN(adj_e)(&g, ones, WE, ec, en);
    FN(adj_h)(&g, ones, cq, E, ec, en);
    if (n_src > 0 && grad_f0 && src_i) FN(record)(grad_f0 + t * S * n_src, E[src_comp], src_i, S, n_src, g.N);
    FN(adj_h)(&g, ca, cq, L, lc, ln);
    if (n_rec > 0 && grad_r && rec_i) FN(inject)(L[rec_comp], grad_r + t * S * n_rec, rec_i, S, n_rec, g.N);
    if (n_src > 0 && grad_df && src_i) FN(record)(grad_df + t * S * n_src, L[src_comp], src_i, S, n_src, g.N);
    for (int m = 0; m < 12; ++m) {
      REAL *tmp = lc[m]; lc[m] = ln[m]; ln[m] = tmp;
      tmp = ec[m]; ec[m] = en[m]; en[m] = tmp;
    }
    if (k > 0 && t % k == 0) {
      const size_t off = (size_t)(t / k) * (size_t)tot * esz;
      FN(image3)(&g, E, store, off, fmt, (REAL)k, grad_ca, shot[0], ca_b);
      FN(image3)(&g, E, store + 3, off, fmt, (REAL)k, grad_cb, shot[1], cb_b);
      FN(image3)(&g, L, dstore, off, fmt, (REAL)k, grad_ca, shot[0], ca_b);
      FN(image3)(&g, L, dstore + 3, off, fmt, (REAL)k, grad_cb, shot[1], cb_b);
      FN(image3)(&g, L, store, off, fmt, (REAL)k, grad_dca, shot[2], ca_b);
      FN(image3)(&g, L, store + 3, off, fmt, (REAL)k, grad_dcb, shot[3], cb_b);
    }
  }
  for (int m = 0; m < 12; ++m) {
    if (lc[m] != lmem[m]) memcpy(lmem[m], lc[m], (size_t)tot * sizeof(REAL));
    if (ec[m] != emem[m]) memcpy(emem[m], ec[m], (size_t)tot * sizeof(REAL));
  }
  REAL *outs[4] = {grad_ca, grad_cb, grad_dca, grad_dcb};
  for (int q = 0; q < 4; ++q) {
    if (!shot[q]) continue;
    for (int64_t j = 0; j < g.N; ++j) {
      REAL sum = 0;
      for (int64_t s = 0; s < S; ++s) sum = sum + shot[q][s * g.N + j];
      outs[q][j] = outs[q][j] + sum;
    }
    free(shot[q]);
  }
  free(scratch);
  free(ones);
  free(w);
}

#undef FN
#undef CAT2
#undef CAT2_
