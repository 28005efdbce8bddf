// 3-D Maxwell (Yee) kernels for stencil orders 4, 6 and 8 (half width
// P = 2, 3, 4): forward H and E half steps (with snapshot storage), the Born
// E half step, and the exact adjoint half steps.  Included by em3d.cu inside
// its namespace, after the order-2 kernels whose helpers (G3, Col, column,
// ccoord, Prof, prof_at, div_k, Snap, Mem12, msz*) it uses.
//
// Differences follow the reference's staggered macros (src/tide/csrc/common/
// staggered_grid.h:31-131 forward, :133-220 transposes): coefficient m of an
// order-2P difference is the literal fraction rounded to T, terms are summed
// from m = 0 up and the sum is scaled by 1 / h once.  The adjoint gathers,
// for each lambda_H (resp. lambda_E) component and each of its two axes, the
// raw terms of the 2P cells the forward difference of that axis reads (zero
// outside the update domain [P, n - P + 1) and, for half-grid terms, on the
// planes c >= n - P), and combines them with the transposed coefficients.
//
// Launch shape: the column march of the order-2 kernels (32 x 8 threads, a
// z run of kZRun cells per thread) over the update domain; operands are read
// straight from global memory through the read-only path, the 2P-wide
// neighbourhoods of adjacent threads and cells meeting in L1 / L2.
#pragma once

template <typename T, int P> __device__ __forceinline__ T fd_coef(int m) {
  if (P == 2) return m == 0 ? (T)(9.0 / 8.0) : (T)(-1.0 / 24.0);
  if (P == 3) return m == 0 ? (T)(75.0 / 64.0) : m == 1 ? (T)(-25.0 / 384.0) : (T)(3.0 / 640.0);
  return m == 0 ? (T)(1225.0 / 1024.0)
         : m == 1 ? (T)(-245.0 / 3072.0)
         : m == 2 ? (T)(49.0 / 5120.0)
                  : (T)(-5.0 / 7168.0);
}

// Integer-grid difference of f at j along stride sd (DIFF?1).
template <typename T, int P>
__device__ __forceinline__ T pd1(const T *__restrict__ f, int64_t j, int64_t sd, T rd) {
  T acc = fd_coef<T, P>(0) * (ld(f + j) - ld(f + j - sd));
#pragma unroll
  for (int m = 1; m < P; ++m)
    acc = acc + fd_coef<T, P>(m) * (ld(f + j + m * sd) - ld(f + j - (m + 1) * sd));
  return acc * rd;
}

// Half-grid difference (DIFF?H1).
template <typename T, int P>
__device__ __forceinline__ T pdh(const T *__restrict__ f, int64_t j, int64_t sd, T rd) {
  T acc = fd_coef<T, P>(0) * (ld(f + j + sd) - ld(f + j));
#pragma unroll
  for (int m = 1; m < P; ++m)
    acc = acc + fd_coef<T, P>(m) * (ld(f + j + (m + 1) * sd) - ld(f + j - m * sd));
  return acc * rd;
}

// Transposed difference over raw terms r[0 .. 2P): coefficient m pairs
// r[P - 1 - m] with r[P + m] (DIFF?1_ADJ / DIFF?H1_ADJ with unit F).
template <typename T, int P> __device__ __forceinline__ T ptadj(const T (&r)[2 * P], T rd) {
  T acc = fd_coef<T, P>(0) * (r[P - 1] * (T)1 - r[P] * (T)1);
#pragma unroll
  for (int m = 1; m < P; ++m) acc = acc + fd_coef<T, P>(m) * (r[P - 1 - m] * (T)1 - r[P + m] * (T)1);
  return acc * rd;
}

// One CPML-corrected derivative: m <- b m + a d, d <- d / k + m.
template <typename T>
__device__ __forceinline__ T cpml(T d, T *__restrict__ mem, int64_t m, const Prof<T> &f) {
  const T v = f.b * mem[m] + f.a * d;
  mem[m] = v;
  return div_k(d, f.k) + v;
}

// Compact in-shot index of (z, y, x) in a memory of `AXIS`.
template <typename T, int AXIS>
__device__ __forceinline__ int64_t pmi(const G3<T> &g, int z, int y, int x) {
  if (AXIS == 0) return ((int64_t)ccoord(z, g.z0, g.zhs) * g.ny + y) * g.nx + x;
  if (AXIS == 1) return ((int64_t)z * g.eyc + ccoord(y, g.y0, g.yhs)) * g.nx + x;
  return ((int64_t)z * g.ny + y) * g.exc + ccoord(x, g.x0, g.xhs);
}

// --------------------------------------------------------------- forward H
template <typename T, int P>
__global__ void __launch_bounds__(256)
k3p_fwd_h(G3<T> g, const T *__restrict__ cq, const T *__restrict__ ex, const T *__restrict__ ey,
          const T *__restrict__ ez, T *__restrict__ hx, T *__restrict__ hy, T *__restrict__ hz,
          T *__restrict__ m_ey_z, T *__restrict__ m_ez_y, T *__restrict__ m_ez_x,
          T *__restrict__ m_ex_z, T *__restrict__ m_ex_y, T *__restrict__ m_ey_x) {
  Col c;
  if (!column(g, c)) return;
  const int nz = g.nz, ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t sz = (int64_t)ny * nx, sy = nx;
  const int64_t base = (int64_t)c.s * g.N;
  ex += base; ey += base; ez += base; hx += base; hy += base; hz += base;
  if (g.cq_b) cq += base;
  m_ey_z += c.s * msz0(g); m_ex_z += c.s * msz0(g);
  m_ez_y += c.s * msz1(g); m_ex_y += c.s * msz1(g);
  m_ez_x += c.s * msz2(g); m_ey_x += c.s * msz2(g);
  const bool yok = y < ny - P, xok = x < nx - P;
  const bool py = y < g.y0 || y >= g.y1h, px = x < g.x0 || x >= g.x1h;
  const Prof<T> fy = prof_at(g, PAYH, PKYH, y, py && yok), fx = prof_at(g, PAXH, PKXH, x, px && xok);
  for (int z = c.zb; z < c.ze; ++z) {
    const int64_t j = ((int64_t)z * ny + y) * nx + x;
    const T q = ld(cq + j);
    T dEy_dz = 0, dEz_dy = 0, dEz_dx = 0, dEx_dz = 0, dEx_dy = 0, dEy_dx = 0;
    if (z < nz - P) {
      dEy_dz = pdh<T, P>(ey, j, sz, g.rdz);
      dEx_dz = pdh<T, P>(ex, j, sz, g.rdz);
      if (z < g.z0 || z >= g.z1h) {
        const Prof<T> fz = prof_at(g, PAZH, PKZH, z, true);
        const int64_t m = pmi<T, 0>(g, z, y, x);
        dEy_dz = cpml(dEy_dz, m_ey_z, m, fz);
        dEx_dz = cpml(dEx_dz, m_ex_z, m, fz);
      }
    }
    if (yok) {
      dEz_dy = pdh<T, P>(ez, j, sy, g.rdy);
      dEx_dy = pdh<T, P>(ex, j, sy, g.rdy);
      if (py) {
        const int64_t m = pmi<T, 1>(g, z, y, x);
        dEz_dy = cpml(dEz_dy, m_ez_y, m, fy);
        dEx_dy = cpml(dEx_dy, m_ex_y, m, fy);
      }
    }
    if (xok) {
      dEz_dx = pdh<T, P>(ez, j, 1, g.rdx);
      dEy_dx = pdh<T, P>(ey, j, 1, g.rdx);
      if (px) {
        const int64_t m = pmi<T, 2>(g, z, y, x);
        dEz_dx = cpml(dEz_dx, m_ez_x, m, fx);
        dEy_dx = cpml(dEy_dx, m_ey_x, m, fx);
      }
    }
    hx[j] = hx[j] - q * (dEy_dz - dEz_dy);
    hy[j] = hy[j] - q * (dEz_dx - dEx_dz);
    hz[j] = hz[j] - q * (dEx_dy - dEy_dx);
  }
}

// Curl of H at cell j with its CPML corrections (the E half step of one state).
template <typename T, int P>
__device__ __forceinline__ void pcurl_h(const G3<T> &g, const T *__restrict__ hx,
                                        const T *__restrict__ hy, const T *__restrict__ hz,
                                        int64_t j, int z, int y, int x, bool pz, bool py, bool px,
                                        const Prof<T> &fz, const Prof<T> &fy, const Prof<T> &fx,
                                        const BornMem<T> &mm, T (&cu)[3]) {
  const int64_t sz = (int64_t)g.ny * g.nx, sy = g.nx;
  T dHy_dz = pd1<T, P>(hy, j, sz, g.rdz);
  T dHz_dy = pd1<T, P>(hz, j, sy, g.rdy);
  T dHz_dx = pd1<T, P>(hz, j, 1, g.rdx);
  T dHx_dz = pd1<T, P>(hx, j, sz, g.rdz);
  T dHx_dy = pd1<T, P>(hx, j, sy, g.rdy);
  T dHy_dx = pd1<T, P>(hy, j, 1, g.rdx);
  if (pz) {
    const int64_t m = pmi<T, 0>(g, z, y, x);
    dHy_dz = cpml(dHy_dz, mm.hy_z, m, fz);
    dHx_dz = cpml(dHx_dz, mm.hx_z, m, fz);
  }
  if (py) {
    const int64_t m = pmi<T, 1>(g, z, y, x);
    dHz_dy = cpml(dHz_dy, mm.hz_y, m, fy);
    dHx_dy = cpml(dHx_dy, mm.hx_y, m, fy);
  }
  if (px) {
    const int64_t m = pmi<T, 2>(g, z, y, x);
    dHz_dx = cpml(dHz_dx, mm.hz_x, m, fx);
    dHy_dx = cpml(dHy_dx, mm.hy_x, m, fx);
  }
  cu[0] = dHy_dz - dHz_dy;
  cu[1] = dHz_dx - dHx_dz;
  cu[2] = dHx_dy - dHy_dx;
}

template <typename T>
__device__ __forceinline__ BornMem<T> shot_mem(const G3<T> &g, BornMem<T> m, int s) {
  const int64_t k0 = s * msz0(g), k1 = s * msz1(g), k2 = s * msz2(g);
  m.hy_z += k0; m.hx_z += k0;
  m.hz_y += k1; m.hx_y += k1;
  m.hz_x += k2; m.hy_x += k2;
  return m;
}

// --------------------------------------------------------------- forward E
template <typename T, typename S, int P>
__global__ void __launch_bounds__(256)
k3p_fwd_e(G3<T> g, const T *__restrict__ ca, const T *__restrict__ cb, T *__restrict__ ex,
          T *__restrict__ ey, T *__restrict__ ez, const T *__restrict__ hx,
          const T *__restrict__ hy, const T *__restrict__ hz, BornMem<T> mm,
          S *__restrict__ st_ex, S *__restrict__ st_ey, S *__restrict__ st_ez,
          S *__restrict__ st_cx, S *__restrict__ st_cy, S *__restrict__ st_cz) {
  Col c;
  if (!column(g, c)) return;
  const int ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t base = (int64_t)c.s * g.N;
  ex += base; ey += base; ez += base; hx += base; hy += base; hz += base;
  if (g.ca_b) ca += base;
  if (g.cb_b) cb += base;
  const bool se = st_ex != nullptr, sc = st_cx != nullptr;
  if (se) { st_ex += base; st_ey += base; st_ez += base; }
  if (sc) { st_cx += base; st_cy += base; st_cz += base; }
  mm = shot_mem(g, mm, c.s);
  const bool py = y < g.y0 || y >= g.y1, px = x < g.x0 || x >= g.x1;
  const Prof<T> fy = prof_at(g, PAY, PKY, y, py), fx = prof_at(g, PAX, PKX, x, px);
  for (int z = c.zb; z < c.ze; ++z) {
    const int64_t j = ((int64_t)z * ny + y) * nx + x;
    const bool pz = z < g.z0 || z >= g.z1;
    const Prof<T> fz = prof_at(g, PAZ, PKZ, z, pz);
    T cu[3];
    pcurl_h<T, P>(g, hx, hy, hz, j, z, y, x, pz, py, px, fz, fy, fx, mm, cu);
    const T e_x = ex[j], e_y = ey[j], e_z = ez[j];
    if (se) {
      st_ex[j] = Snap<S, T>::enc(e_x);
      st_ey[j] = Snap<S, T>::enc(e_y);
      st_ez[j] = Snap<S, T>::enc(e_z);
    }
    if (sc) {
      st_cx[j] = Snap<S, T>::enc(cu[0]);
      st_cy[j] = Snap<S, T>::enc(cu[1]);
      st_cz[j] = Snap<S, T>::enc(cu[2]);
    }
    const T a = ld(ca + j), b = ld(cb + j);
    ex[j] = a * e_x + b * cu[0];
    ey[j] = a * e_y + b * cu[1];
    ez[j] = a * e_z + b * cu[2];
  }
}

// Born E half step (maxwell_3d_inst.cpp:1390-1475) at orders 4 to 8.
template <typename T, typename S, int P>
__global__ void __launch_bounds__(256)
k3p_born_e(G3<T> g, const T *__restrict__ ca, const T *__restrict__ cb,
           const T *__restrict__ dca, const T *__restrict__ dcb, T *__restrict__ ex,
           T *__restrict__ ey, T *__restrict__ ez, const T *__restrict__ hx,
           const T *__restrict__ hy, const T *__restrict__ hz, T *__restrict__ dex,
           T *__restrict__ dey, T *__restrict__ dez, const T *__restrict__ dhx,
           const T *__restrict__ dhy, const T *__restrict__ dhz, BornMem<T> mb, BornMem<T> ms,
           BornSnap<S> sn) {
  Col c;
  if (!column(g, c)) return;
  const int ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t base = (int64_t)c.s * g.N;
  ex += base; ey += base; ez += base; hx += base; hy += base; hz += base;
  dex += base; dey += base; dez += base; dhx += base; dhy += base; dhz += base;
  if (g.ca_b) { ca += base; dca += base; }
  if (g.cb_b) { cb += base; dcb += base; }
  mb = shot_mem(g, mb, c.s);
  ms = shot_mem(g, ms, c.s);
  const bool py = y < g.y0 || y >= g.y1, px = x < g.x0 || x >= g.x1;
  const Prof<T> fy = prof_at(g, PAY, PKY, y, py), fx = prof_at(g, PAX, PKX, x, px);
  for (int z = c.zb; z < c.ze; ++z) {
    const int64_t j = ((int64_t)z * ny + y) * nx + x;
    const bool pz = z < g.z0 || z >= g.z1;
    const Prof<T> fz = prof_at(g, PAZ, PKZ, z, pz);
    T cu[2][3];
    pcurl_h<T, P>(g, hx, hy, hz, j, z, y, x, pz, py, px, fz, fy, fx, mb, cu[0]);
    pcurl_h<T, P>(g, dhx, dhy, dhz, j, z, y, x, pz, py, px, fz, fy, fx, ms, cu[1]);
    const T a = ld(ca + j), b = ld(cb + j), da = ld(dca + j), db = ld(dcb + j);
    T *E[3] = {ex, ey, ez}, *D[3] = {dex, dey, dez};
    born_store(sn, base + j, E, D, cu, j);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T e_old = E[k][j];
      D[k][j] = a * D[k][j] + b * cu[1][k] + da * e_old + db * cu[0][k];
      E[k][j] = a * e_old + b * cu[0][k];
    }
  }
}

// ---------------------------------------------------------------- adjoint
// Raw adjoint term of the cell (z, y, x) on the axis AXIS (reference
// raw_e_side / raw_h_side): zero outside the update domain (and for half-grid
// terms on the planes c >= n - P); q = +-coef lambda; in the CPML strip of
// the axis a (b m + q) + q / kappa with m the current memory adjoint.
template <typename T, int AXIS, bool HALF>
__device__ __forceinline__ T praw(const G3<T> &g, const T *__restrict__ coef,
                                  const T *__restrict__ lam, const T *__restrict__ mem, bool neg,
                                  int z, int y, int x, int64_t j) {
  const int cc = AXIS == 0 ? z : AXIS == 1 ? y : x;
  const int n = AXIS == 0 ? g.nz : AXIS == 1 ? g.ny : g.nx;
  if (cc < g.P || cc >= n - g.P + (HALF ? 0 : 1)) return (T)0;
  T q = ld(coef + j) * ld(lam + j);
  if (neg) q = -q;
  const int lo = AXIS == 0 ? g.z0 : AXIS == 1 ? g.y0 : g.x0;
  const int hi = HALF ? (AXIS == 0 ? g.z1h : AXIS == 1 ? g.y1h : g.x1h)
                      : (AXIS == 0 ? g.z1 : AXIS == 1 ? g.y1 : g.x1);
  if (!(cc < lo || cc >= hi)) return q;
  const int pa = HALF ? (AXIS == 0 ? PAZH : AXIS == 1 ? PAYH : PAXH)
                      : (AXIS == 0 ? PAZ : AXIS == 1 ? PAY : PAX);
  const int pk = HALF ? (AXIS == 0 ? PKZH : AXIS == 1 ? PKYH : PKXH)
                      : (AXIS == 0 ? PKZ : AXIS == 1 ? PKY : PKX);
  const T A = ld(g.p[pa] + cc), B = ld(g.p[pa + 1] + cc), K = ld(g.p[pk] + cc);
  const T m_used = B * ld(mem + pmi<T, AXIS>(g, z, y, x)) + q;
  return A * m_used + q / K;
}

// Raw terms of the 2P cells at offsets o0 .. o0 + 2P - 1 along AXIS from
// (z, y, x), combined by the transposed difference.
template <typename T, int P, int AXIS, bool HALF>
__device__ __forceinline__ T pgather(const G3<T> &g, const T *__restrict__ coef,
                                     const T *__restrict__ lam, const T *__restrict__ mem,
                                     bool neg, int z, int y, int x, int64_t j, T rd) {
  constexpr int o0 = HALF ? -P : 1 - P;
  const int64_t sd = AXIS == 0 ? (int64_t)g.ny * g.nx : AXIS == 1 ? (int64_t)g.nx : 1;
  T r[2 * P];
#pragma unroll
  for (int k = 0; k < 2 * P; ++k) {
    const int o = o0 + k;
    r[k] = praw<T, AXIS, HALF>(g, coef, lam, mem, neg, z + (AXIS == 0 ? o : 0),
                               y + (AXIS == 1 ? o : 0), x + (AXIS == 2 ? o : 0), j + o * sd);
  }
  return ptadj<T, P>(r, rd);
}

// Adjoint of the forward E update: next E-phase memory adjoints at the own
// cell (in their strips) and lambda_H += transposed differences of the raw
// terms of lambda_E's neighbourhood.
template <typename T, typename S, int P>
__global__ void __launch_bounds__(256)
k3p_adj_e(G3<T> g, const T *__restrict__ cb, const T *__restrict__ lex,
          const T *__restrict__ ley, const T *__restrict__ lez, T *__restrict__ lhx,
          T *__restrict__ lhy, T *__restrict__ lhz, Mem12<T> cur, Mem12<T> nxt,
          GradFold<T, S> gf) {
  Col c;
  if (!column(g, c)) return;
  const int ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t base = (int64_t)c.s * g.N;
  lex += base; ley += base; lez += base; lhx += base; lhy += base; lhz += base;
  if (g.cb_b) cb += base;
  const int64_t k0 = c.s * msz0(g), k1 = c.s * msz1(g), k2 = c.s * msz2(g);
  const T *c_hy_z = cur.m[LHY_Z] + k0, *c_hx_z = cur.m[LHX_Z] + k0;
  const T *c_hz_y = cur.m[LHZ_Y] + k1, *c_hx_y = cur.m[LHX_Y] + k1;
  const T *c_hz_x = cur.m[LHZ_X] + k2, *c_hy_x = cur.m[LHY_X] + k2;
  const bool py = y < g.y0 || y >= g.y1, px = x < g.x0 || x >= g.x1;
  const T by = py ? ld(g.p[PBY] + y) : (T)0, bx = px ? ld(g.p[PBX] + x) : (T)0;
  for (int z = c.zb; z < c.ze; ++z) {
    const int64_t j = ((int64_t)z * ny + y) * nx + x;
    const T b = ld(cb + j);
    const T lx = ld(lex + j), ly = ld(ley + j), lz = ld(lez + j);
    const T qx = b * lx, qy = b * ly, qz = b * lz;
    fold_grad(g, gf, base + j, j, lx, ly, lz);
    if (z < g.z0 || z >= g.z1) {
      const int64_t m = pmi<T, 0>(g, z, y, x);
      const T bz = ld(g.p[PBZ] + z);
      nxt.m[LHY_Z][k0 + m] = bz * ld(c_hy_z + m) + qx;
      nxt.m[LHX_Z][k0 + m] = bz * ld(c_hx_z + m) - qy;
    }
    if (py) {
      const int64_t m = pmi<T, 1>(g, z, y, x);
      nxt.m[LHZ_Y][k1 + m] = by * ld(c_hz_y + m) - qx;
      nxt.m[LHX_Y][k1 + m] = by * ld(c_hx_y + m) + qz;
    }
    if (px) {
      const int64_t m = pmi<T, 2>(g, z, y, x);
      nxt.m[LHZ_X][k2 + m] = bx * ld(c_hz_x + m) + qy;
      nxt.m[LHY_X][k2 + m] = bx * ld(c_hy_x + m) - qz;
    }
    const T a1 = pgather<T, P, 0, false>(g, cb, ley, c_hx_z, true, z, y, x, j, g.rdz);
    const T a2 = pgather<T, P, 1, false>(g, cb, lez, c_hx_y, false, z, y, x, j, g.rdy);
    lhx[j] = lhx[j] + (a1 + a2);
    const T b1 = pgather<T, P, 0, false>(g, cb, lex, c_hy_z, false, z, y, x, j, g.rdz);
    const T b2 = pgather<T, P, 2, false>(g, cb, lez, c_hy_x, true, z, y, x, j, g.rdx);
    lhy[j] = lhy[j] + (b1 + b2);
    const T c1 = pgather<T, P, 1, false>(g, cb, lex, c_hz_y, true, z, y, x, j, g.rdy);
    const T c2 = pgather<T, P, 2, false>(g, cb, ley, c_hz_x, false, z, y, x, j, g.rdx);
    lhz[j] = lhz[j] + (c1 + c2);
  }
}

// Adjoint of the forward H update: next H-phase memory adjoints at the own
// cell (in their strips; none on the planes c >= n - P) and lambda_E <-
// ca lambda_E + transposed differences of the raw terms of lambda_H's
// neighbourhood.
template <typename T, int P>
__global__ void __launch_bounds__(256)
k3p_adj_h(G3<T> g, const T *__restrict__ ca, const T *__restrict__ cq,
          const T *__restrict__ lhx, const T *__restrict__ lhy, const T *__restrict__ lhz,
          T *__restrict__ lex, T *__restrict__ ley, T *__restrict__ lez, Mem12<T> cur,
          Mem12<T> nxt) {
  Col c;
  if (!column(g, c)) return;
  const int nz = g.nz, ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t base = (int64_t)c.s * g.N;
  lhx += base; lhy += base; lhz += base; lex += base; ley += base; lez += base;
  if (g.ca_b) ca += base;
  if (g.cq_b) cq += base;
  const int64_t k0 = c.s * msz0(g), k1 = c.s * msz1(g), k2 = c.s * msz2(g);
  const T *c_ey_z = cur.m[LEY_Z] + k0, *c_ex_z = cur.m[LEX_Z] + k0;
  const T *c_ez_y = cur.m[LEZ_Y] + k1, *c_ex_y = cur.m[LEX_Y] + k1;
  const T *c_ez_x = cur.m[LEZ_X] + k2, *c_ey_x = cur.m[LEY_X] + k2;
  const bool py = y < ny - P && (y < g.y0 || y >= g.y1h);
  const bool px = x < nx - P && (x < g.x0 || x >= g.x1h);
  const T by = py ? ld(g.p[PBYH] + y) : (T)0, bx = px ? ld(g.p[PBXH] + x) : (T)0;
  for (int z = c.zb; z < c.ze; ++z) {
    const int64_t j = ((int64_t)z * ny + y) * nx + x;
    const T q = ld(cq + j);
    const T l_hx = ld(lhx + j), l_hy = ld(lhy + j), l_hz = ld(lhz + j);
    if (z < nz - P && (z < g.z0 || z >= g.z1h)) {
      const int64_t m = pmi<T, 0>(g, z, y, x);
      const T bz = ld(g.p[PBZH] + z);
      nxt.m[LEY_Z][k0 + m] = bz * ld(c_ey_z + m) - q * l_hx;
      nxt.m[LEX_Z][k0 + m] = bz * ld(c_ex_z + m) + q * l_hy;
    }
    if (py) {
      const int64_t m = pmi<T, 1>(g, z, y, x);
      nxt.m[LEZ_Y][k1 + m] = by * ld(c_ez_y + m) + q * l_hx;
      nxt.m[LEX_Y][k1 + m] = by * ld(c_ex_y + m) - q * l_hz;
    }
    if (px) {
      const int64_t m = pmi<T, 2>(g, z, y, x);
      nxt.m[LEZ_X][k2 + m] = bx * ld(c_ez_x + m) - q * l_hy;
      nxt.m[LEY_X][k2 + m] = bx * ld(c_ey_x + m) + q * l_hz;
    }
    const T a = ld(ca + j);
    const T v_x = a * lex[j], v_y = a * ley[j], v_z = a * lez[j];
    const T e1 = pgather<T, P, 0, true>(g, cq, lhx, c_ey_z, true, z, y, x, j, g.rdz);
    const T e2 = pgather<T, P, 2, true>(g, cq, lhz, c_ey_x, false, z, y, x, j, g.rdx);
    ley[j] = v_y + (e1 + e2);
    const T f1 = pgather<T, P, 0, true>(g, cq, lhy, c_ex_z, false, z, y, x, j, g.rdz);
    const T f2 = pgather<T, P, 1, true>(g, cq, lhz, c_ex_y, true, z, y, x, j, g.rdy);
    lex[j] = v_x + (f1 + f2);
    const T h1 = pgather<T, P, 1, true>(g, cq, lhx, c_ez_y, false, z, y, x, j, g.rdy);
    const T h2 = pgather<T, P, 2, true>(g, cq, lhy, c_ez_x, true, z, y, x, j, g.rdx);
    lez[j] = v_z + (h1 + h2);
  }
}
