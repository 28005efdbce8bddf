// 3-D Maxwell (Yee) path, stencil orders 2, 4, 6 and 8: forward, forward
// with snapshot storage, Born forward and exact adjoint with coefficient
// gradients, behind the reference's maxwell_3d_{S}_{float,double}_{forward,
// forward_with_storage,born_forward,backward}_cuda symbols (declared in
// include/tide_b200.h).  Order 2 has the register-marching kernels below;
// orders 4 to 8 the generic kernels of em3d_hi.cuh.
//
// Arithmetic follows the reference's 3-D update and adjoint (forward H/E
// src/tide/csrc/em3d/maxwell_3d_inst.cpp:560-702; snapshots
// maxwell_3d_cuda_inst.cu:755-868; adjoint :1478-1829; coefficient gradient
// :2301-2368; shot reduction :2713-2727; conversion :2729-2776), with IEEE
// division by kappa everywhere (the reference CPU backend and its storing CUDA
// kernel divide; its plain CUDA forward multiplies by a reciprocal), so the
// forward is bit-identical to the reference CPU backend.
//
// Layout: fields [S, nz, ny, nx]; CPML memories compacted along their own
// axis (cells c < c0 and c >= max(c0, c1 - 1) kept) as the reference's CUDA
// callers allocate them.  Launch: blocks of 32 (x) x kBlockY3 (y) threads,
// each thread marching kZRun consecutive z cells of one (y, x) column; grid
// z = shot x z-run.  On the 153^3 x 4-shot grid, 32 x 4 blocks and 8-cell
// runs measured 6% faster per fwd+adj than 32 x 8 and 16 (bit-identical).  Along the march the z neighbour of a cell (fields, and in
// the adjoint the raw CPML terms) is carried in registers from the previous
// cell; per-thread pointers start at the thread's shot, and the y / x strip
// state and profile values of a column are read once.  CPML memories are
// read and written only in their strips (the compact planes outside the
// update domain stay zero).
#include <algorithm>
#include <utility>
#include <vector>

#include <cuda_bf16.h>

#include "../../include/tide_b200.h"
#include "tb_common.cuh"
#include "tb_store.cuh"

namespace tb {
namespace {

constexpr int kZRun = 8;
constexpr int kBlockY3 = 4;

enum { PAZ, PBZ, PAZH, PBZH, PAY, PBY, PAYH, PBYH, PAX, PBX, PAXH, PBXH,
       PKZ, PKZH, PKY, PKYH, PKX, PKXH, kNProf };

template <typename T> struct G3 {
  const T *p[kNProf];
  T rdz, rdy, rdx;
  int nz, ny, nx, S;
  int64_t N;
  int z0, y0, x0, z1, y1, x1, z1h, y1h, x1h;
  int zhs, yhs, xhs;  // first kept cell of each axis's upper strip (compact layout)
  int ezc, eyc, exc;  // memory extents along z, y, x
  int P;              // half stencil width: update domain [P, n - P + 1) per axis
  bool ca_b, cb_b, cq_b;
};

template <typename T> __device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// d / k for a CPML kappa k > 0; a zero numerator (a field the wave has not
// reached) divides 1 instead so the division stays on its fast path, and d
// itself (= d / k, sign included) is returned.
template <typename T> __device__ __forceinline__ T div_k(T d, T k) {
  const T q = (d == (T)0 ? (T)1 : d) / k;
  return d == (T)0 ? d : q;
}

template <typename S, typename T> struct Snap {
  __device__ static S enc(T v) { return (S)v; }
  __device__ static T dec(S v) { return (T)v; }
};
template <typename T> struct Snap<__nv_bfloat16, T> {
  __device__ static __nv_bfloat16 enc(T v) { return __float2bfloat16((float)v); }
  __device__ static T dec(__nv_bfloat16 v) { return (T)__bfloat162float(v); }
};

struct Cell {
  int s, z, y, x, zend;
  int64_t i, j;  // flat index with and without the shot offset
};
template <typename T>
__device__ __forceinline__ bool first_cell(const G3<T> &g, Cell &c) {
  const int zruns = (g.nz + kZRun - 1) / kZRun;
  c.x = blockIdx.x * blockDim.x + threadIdx.x;
  c.y = blockIdx.y * blockDim.y + threadIdx.y;
  c.s = blockIdx.z / zruns;
  c.z = (blockIdx.z - c.s * zruns) * kZRun;
  c.zend = min(c.z + kZRun, g.nz - g.P + 1);
  if (c.x < g.P || c.x >= g.nx - g.P + 1 || c.y < g.P || c.y >= g.ny - g.P + 1) return false;
  if (c.z < g.P) c.z = g.P;
  return c.z < c.zend;
}
__device__ __forceinline__ void set_index(Cell &c, int ny, int nx, int64_t N) {
  c.j = ((int64_t)c.z * ny + c.y) * nx + c.x;
  c.i = (int64_t)c.s * N + c.j;
}

// ---------------------------------------------------------------- forward
// Column of one thread: shot s, (y, x) and the z run [zb, ze) of cells in
// the update domain (z, y, x in [P, n - P + 1)).
struct Col {
  int s, y, x, zb, ze;
};
template <typename T>
__device__ __forceinline__ bool column(const G3<T> &g, Col &c) {
  const int zruns = (g.nz + kZRun - 1) / kZRun;
  c.x = blockIdx.x * blockDim.x + threadIdx.x;
  c.y = blockIdx.y * blockDim.y + threadIdx.y;
  c.s = blockIdx.z / zruns;
  c.zb = (blockIdx.z - c.s * zruns) * kZRun;
  c.ze = min(c.zb + kZRun, g.nz - g.P + 1);
  if (c.x < g.P || c.x >= g.nx - g.P + 1 || c.y < g.P || c.y >= g.ny - g.P + 1) return false;
  if (c.zb < g.P) c.zb = g.P;
  return c.zb < c.ze;
}

// Memory coordinate of a strip cell c along an axis whose memories keep the
// cells c < lo and c >= hs: the compact layout of the forward and adjoint
// entry points has hs = max(lo, hi - 1), the full layout of the Born entry
// points hs = lo (identity).
__device__ __forceinline__ int ccoord(int c, int lo, int hs) {
  return c < lo ? c : lo + c - hs;
}

// Per-shot element counts of the compact memories along z, y, x.
template <typename T> __device__ __forceinline__ int64_t msz0(const G3<T> &g) {
  return (int64_t)g.ezc * g.ny * g.nx;
}
template <typename T> __device__ __forceinline__ int64_t msz1(const G3<T> &g) {
  return (int64_t)g.nz * g.eyc * g.nx;
}
template <typename T> __device__ __forceinline__ int64_t msz2(const G3<T> &g) {
  return (int64_t)g.nz * g.ny * g.exc;
}

// CPML profile triple (a, b, kappa) of one coordinate.
template <typename T> struct Prof {
  T a, b, k;
};
template <typename T>
__device__ __forceinline__ Prof<T> prof_at(const G3<T> &g, int pa, int pk, int c, bool on) {
  if (!on) return Prof<T>{(T)0, (T)0, (T)1};
  return Prof<T>{ld(g.p[pa] + c), ld(g.p[pa + 1] + c), ld(g.p[pk] + c)};
}

// Operands of one forward-H cell, loaded one cell ahead of its arithmetic so
// that two cells' loads are in flight per thread.
template <typename T> struct OpsH {
  T q, e_z, n_x, n_y, ez_y, ex_y, ez_x, ey_x, h_x, h_y, h_z;
};

template <typename T>
__global__ void __launch_bounds__(256, 4)
k3_fwd_h(G3<T> g, const T *__restrict__ cq, const T *__restrict__ ex, const T *__restrict__ ey,
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
  const bool yok = y < ny - 1, xok = x < nx - 1;
  const bool py = y < g.y0 || y >= g.y1h, px = x < g.x0 || x >= g.x1h;
  const Prof<T> fy = prof_at(g, PAYH, PKYH, y, py && yok), fx = prof_at(g, PAXH, PKXH, x, px && xok);
  const int64_t o1 = (int64_t)ccoord(y, g.y0, g.yhs) * nx + x, s1 = (int64_t)g.eyc * nx;
  const int64_t o2 = (int64_t)y * g.exc + ccoord(x, g.x0, g.xhs), s2 = (int64_t)ny * g.exc;
  auto load = [&](int z, int64_t jj) {
    OpsH<T> o{};
    o.q = ld(cq + jj);
    o.e_z = ld(ez + jj);
    if (z < nz - 1) {
      o.n_y = ld(ey + jj + sz);
      o.n_x = ld(ex + jj + sz);
    }
    if (yok) {
      o.ez_y = ld(ez + jj + sy);
      o.ex_y = ld(ex + jj + sy);
    }
    if (xok) {
      o.ez_x = ld(ez + jj + 1);
      o.ey_x = ld(ey + jj + 1);
    }
    o.h_x = hx[jj];
    o.h_y = hy[jj];
    o.h_z = hz[jj];
    return o;
  };
  int64_t j = ((int64_t)c.zb * ny + y) * nx + x;
  T e_x = ld(ex + j), e_y = ld(ey + j);
  OpsH<T> o = load(c.zb, j);
  for (int z = c.zb; z < c.ze; ++z, j += sz) {
    OpsH<T> on{};
    if (z + 1 < c.ze) on = load(z + 1, j + sz);
    T dEy_dz = 0, dEz_dy = 0, dEz_dx = 0, dEx_dz = 0, dEx_dy = 0, dEy_dx = 0;
    if (z < nz - 1) {
      T d = (o.n_y - e_y) * g.rdz;
      T d2 = (o.n_x - e_x) * g.rdz;
      if (z < g.z0 || z >= g.z1h) {
        const int64_t m = ((int64_t)ccoord(z, g.z0, g.zhs) * ny + y) * nx + x;
        const T b = ld(g.p[PBZH] + z), a = ld(g.p[PAZH] + z), k = ld(g.p[PKZH] + z);
        const T m1 = b * m_ey_z[m] + a * d;
        m_ey_z[m] = m1;
        d = div_k(d, k) + m1;
        const T m2 = b * m_ex_z[m] + a * d2;
        m_ex_z[m] = m2;
        d2 = div_k(d2, k) + m2;
      }
      dEy_dz = d;
      dEx_dz = d2;
    }
    if (yok) {
      T d = (o.ez_y - o.e_z) * g.rdy;
      T d2 = (o.ex_y - e_x) * g.rdy;
      if (py) {
        const int64_t m = z * s1 + o1;
        const T m1 = fy.b * m_ez_y[m] + fy.a * d;
        m_ez_y[m] = m1;
        d = div_k(d, fy.k) + m1;
        const T m2 = fy.b * m_ex_y[m] + fy.a * d2;
        m_ex_y[m] = m2;
        d2 = div_k(d2, fy.k) + m2;
      }
      dEz_dy = d;
      dEx_dy = d2;
    }
    if (xok) {
      T d = (o.ez_x - o.e_z) * g.rdx;
      T d2 = (o.ey_x - e_y) * g.rdx;
      if (px) {
        const int64_t m = z * s2 + o2;
        const T m1 = fx.b * m_ez_x[m] + fx.a * d;
        m_ez_x[m] = m1;
        d = div_k(d, fx.k) + m1;
        const T m2 = fx.b * m_ey_x[m] + fx.a * d2;
        m_ey_x[m] = m2;
        d2 = div_k(d2, fx.k) + m2;
      }
      dEz_dx = d;
      dEy_dx = d2;
    }
    hx[j] = o.h_x - o.q * (dEy_dz - dEz_dy);
    hy[j] = o.h_y - o.q * (dEz_dx - dEx_dz);
    hz[j] = o.h_z - o.q * (dEx_dy - dEy_dx);
    e_x = o.n_x;
    e_y = o.n_y;
    o = on;
  }
}

// Operands of one forward-E cell (loaded one cell ahead, as OpsH).
template <typename T> struct OpsE {
  T a, b, h_x, h_y, h_z, hz_y, hz_x, hx_y, hy_x, e_x, e_y, e_z;
};

template <typename T, typename S>
__global__ void __launch_bounds__(256, 4)
k3_fwd_e(G3<T> g, const T *__restrict__ ca, const T *__restrict__ cb, T *__restrict__ ex,
         T *__restrict__ ey, T *__restrict__ ez, const T *__restrict__ hx,
         const T *__restrict__ hy, const T *__restrict__ hz, T *__restrict__ m_hz_y,
         T *__restrict__ m_hy_z, T *__restrict__ m_hx_z, T *__restrict__ m_hz_x,
         T *__restrict__ m_hy_x, T *__restrict__ m_hx_y, S *__restrict__ st_ex,
         S *__restrict__ st_ey, S *__restrict__ st_ez, S *__restrict__ st_cx,
         S *__restrict__ st_cy, S *__restrict__ st_cz) {
  Col c;
  if (!column(g, c)) return;
  const int ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t sz = (int64_t)ny * nx, sy = nx;
  const int64_t base = (int64_t)c.s * g.N;
  ex += base; ey += base; ez += base; hx += base; hy += base; hz += base;
  if (g.ca_b) ca += base;
  if (g.cb_b) cb += base;
  const bool se = st_ex != nullptr, sc = st_cx != nullptr;
  if (se) { st_ex += base; st_ey += base; st_ez += base; }
  if (sc) { st_cx += base; st_cy += base; st_cz += base; }
  m_hy_z += c.s * msz0(g); m_hx_z += c.s * msz0(g);
  m_hz_y += c.s * msz1(g); m_hx_y += c.s * msz1(g);
  m_hz_x += c.s * msz2(g); m_hy_x += c.s * msz2(g);
  const bool py = y < g.y0 || y >= g.y1, px = x < g.x0 || x >= g.x1;
  const Prof<T> fy = prof_at(g, PAY, PKY, y, py), fx = prof_at(g, PAX, PKX, x, px);
  const int64_t o1 = (int64_t)ccoord(y, g.y0, g.yhs) * nx + x, s1 = (int64_t)g.eyc * nx;
  const int64_t o2 = (int64_t)y * g.exc + ccoord(x, g.x0, g.xhs), s2 = (int64_t)ny * g.exc;
  auto load = [&](int64_t jj) {
    OpsE<T> o;
    o.a = ld(ca + jj);
    o.b = ld(cb + jj);
    o.h_x = ld(hx + jj);
    o.h_y = ld(hy + jj);
    o.h_z = ld(hz + jj);
    o.hz_y = ld(hz + jj - sy);
    o.hz_x = ld(hz + jj - 1);
    o.hx_y = ld(hx + jj - sy);
    o.hy_x = ld(hy + jj - 1);
    o.e_x = ex[jj];
    o.e_y = ey[jj];
    o.e_z = ez[jj];
    return o;
  };
  int64_t j = ((int64_t)c.zb * ny + y) * nx + x;
  T p_x = ld(hx + j - sz), p_y = ld(hy + j - sz);  // Hx, Hy at z - 1
  OpsE<T> o = load(j);
  for (int z = c.zb; z < c.ze; ++z, j += sz) {
    OpsE<T> on{};
    if (z + 1 < c.ze) on = load(j + sz);
    T dHy_dz = (o.h_y - p_y) * g.rdz;
    T dHz_dy = (o.h_z - o.hz_y) * g.rdy;
    T dHz_dx = (o.h_z - o.hz_x) * g.rdx;
    T dHx_dz = (o.h_x - p_x) * g.rdz;
    T dHx_dy = (o.h_x - o.hx_y) * g.rdy;
    T dHy_dx = (o.h_y - o.hy_x) * g.rdx;
    if (z < g.z0 || z >= g.z1) {
      const int64_t m = ((int64_t)ccoord(z, g.z0, g.zhs) * ny + y) * nx + x;
      const T bb = ld(g.p[PBZ] + z), aa = ld(g.p[PAZ] + z), k = ld(g.p[PKZ] + z);
      const T m1 = bb * m_hy_z[m] + aa * dHy_dz;
      m_hy_z[m] = m1;
      dHy_dz = div_k(dHy_dz, k) + m1;
      const T m2 = bb * m_hx_z[m] + aa * dHx_dz;
      m_hx_z[m] = m2;
      dHx_dz = div_k(dHx_dz, k) + m2;
    }
    if (py) {
      const int64_t m = z * s1 + o1;
      const T m1 = fy.b * m_hz_y[m] + fy.a * dHz_dy;
      m_hz_y[m] = m1;
      dHz_dy = div_k(dHz_dy, fy.k) + m1;
      const T m2 = fy.b * m_hx_y[m] + fy.a * dHx_dy;
      m_hx_y[m] = m2;
      dHx_dy = div_k(dHx_dy, fy.k) + m2;
    }
    if (px) {
      const int64_t m = z * s2 + o2;
      const T m1 = fx.b * m_hz_x[m] + fx.a * dHz_dx;
      m_hz_x[m] = m1;
      dHz_dx = div_k(dHz_dx, fx.k) + m1;
      const T m2 = fx.b * m_hy_x[m] + fx.a * dHy_dx;
      m_hy_x[m] = m2;
      dHy_dx = div_k(dHy_dx, fx.k) + m2;
    }
    const T cx = dHy_dz - dHz_dy, cy = dHz_dx - dHx_dz, cz = dHx_dy - dHy_dx;
    if (se) {
      st_ex[j] = Snap<S, T>::enc(o.e_x);
      st_ey[j] = Snap<S, T>::enc(o.e_y);
      st_ez[j] = Snap<S, T>::enc(o.e_z);
    }
    if (sc) {
      st_cx[j] = Snap<S, T>::enc(cx);
      st_cy[j] = Snap<S, T>::enc(cy);
      st_cz[j] = Snap<S, T>::enc(cz);
    }
    ex[j] = o.a * o.e_x + o.b * cx;
    ey[j] = o.a * o.e_y + o.b * cy;
    ez[j] = o.a * o.e_z + o.b * cz;
    p_x = o.h_x;
    p_y = o.h_y;
    o = on;
  }
}

// Born E half-step (maxwell_3d_inst.cpp:1390-1475): background and scattered
// curls with their own CPML memories, then the scattered update
// ca dE + cb dcurl + dca E^n + dcb curl H^n and the background update.  The
// same z-marching columns as k3_fwd_e; H at z - 1 of both states is carried
// in registers.
template <typename T>
struct BornMem {
  T *hz_y, *hy_z, *hx_z, *hz_x, *hy_x, *hx_y;  // E-phase memories of one state
};
// Snapshots one Born E half step stores (maxwell_3d_cuda_inst.cu:1291-1340),
// each [S, nz, ny, nx] of the step or null: background E^n and curl H^n, then
// scattered E^n and curl.
template <typename S> struct BornSnap {
  S *e[3], *c[3], *de[3], *dc[3];
};
template <typename S, typename T>
__device__ __forceinline__ void born_store(const BornSnap<S> &sn, int64_t i, T *const E[3],
                                           T *const D[3], const T (&cu)[2][3], int64_t j) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (sn.e[0]) sn.e[k][i] = Snap<S, T>::enc(E[k][j]);
    if (sn.c[0]) sn.c[k][i] = Snap<S, T>::enc(cu[0][k]);
    if (sn.de[0]) sn.de[k][i] = Snap<S, T>::enc(D[k][j]);
    if (sn.dc[0]) sn.dc[k][i] = Snap<S, T>::enc(cu[1][k]);
  }
}
template <typename T, typename S>
__global__ void __launch_bounds__(256)
k3_born_e(G3<T> g, const T *__restrict__ ca, const T *__restrict__ cb,
          const T *__restrict__ dca, const T *__restrict__ dcb, T *__restrict__ ex,
          T *__restrict__ ey, T *__restrict__ ez, const T *__restrict__ hx,
          const T *__restrict__ hy, const T *__restrict__ hz, T *__restrict__ dex,
          T *__restrict__ dey, T *__restrict__ dez, const T *__restrict__ dhx,
          const T *__restrict__ dhy, const T *__restrict__ dhz, BornMem<T> mb, BornMem<T> ms,
          BornSnap<S> sn) {
  Col c;
  if (!column(g, c)) return;
  const int ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t sz = (int64_t)ny * nx, sy = nx;
  const int64_t base = (int64_t)c.s * g.N;
  ex += base; ey += base; ez += base; hx += base; hy += base; hz += base;
  dex += base; dey += base; dez += base; dhx += base; dhy += base; dhz += base;
  if (g.ca_b) { ca += base; dca += base; }
  if (g.cb_b) { cb += base; dcb += base; }
  const int64_t k0 = c.s * msz0(g), k1 = c.s * msz1(g), k2 = c.s * msz2(g);
  BornMem<T> m[2] = {mb, ms};
  for (int w = 0; w < 2; ++w) {
    m[w].hy_z += k0; m[w].hx_z += k0;
    m[w].hz_y += k1; m[w].hx_y += k1;
    m[w].hz_x += k2; m[w].hy_x += k2;
  }
  const bool py = y < g.y0 || y >= g.y1, px = x < g.x0 || x >= g.x1;
  const Prof<T> fy = prof_at(g, PAY, PKY, y, py), fx = prof_at(g, PAX, PKX, x, px);
  const int64_t o1 = (int64_t)ccoord(y, g.y0, g.yhs) * nx + x, s1 = (int64_t)g.eyc * nx;
  const int64_t o2 = (int64_t)y * g.exc + ccoord(x, g.x0, g.xhs), s2 = (int64_t)ny * g.exc;
  const T *H[2][3] = {{hx, hy, hz}, {dhx, dhy, dhz}};
  int64_t j = ((int64_t)c.zb * ny + y) * nx + x;
  T p_x[2], p_y[2];  // Hx, Hy at z - 1 of both states
  for (int w = 0; w < 2; ++w) {
    p_x[w] = ld(H[w][0] + j - sz);
    p_y[w] = ld(H[w][1] + j - sz);
  }
  for (int z = c.zb; z < c.ze; ++z, j += sz) {
    const T a = ld(ca + j), b = ld(cb + j), da = ld(dca + j), db = ld(dcb + j);
    const bool pz = z < g.z0 || z >= g.z1;
    Prof<T> fz{(T)0, (T)0, (T)1};
    if (pz) fz = prof_at(g, PAZ, PKZ, z, true);
    const int64_t m0 = ((int64_t)ccoord(z, g.z0, g.zhs) * ny + y) * nx + x;
    T cu[2][3];
#pragma unroll
    for (int w = 0; w < 2; ++w) {
      const T h_x = ld(H[w][0] + j), h_y = ld(H[w][1] + j), h_z = ld(H[w][2] + j);
      T dHy_dz = (h_y - p_y[w]) * g.rdz;
      T dHz_dy = (h_z - ld(H[w][2] + j - sy)) * g.rdy;
      T dHz_dx = (h_z - ld(H[w][2] + j - 1)) * g.rdx;
      T dHx_dz = (h_x - p_x[w]) * g.rdz;
      T dHx_dy = (h_x - ld(H[w][0] + j - sy)) * g.rdy;
      T dHy_dx = (h_y - ld(H[w][1] + j - 1)) * g.rdx;
      if (pz) {
        const T m1 = fz.b * m[w].hy_z[m0] + fz.a * dHy_dz;
        m[w].hy_z[m0] = m1;
        dHy_dz = div_k(dHy_dz, fz.k) + m1;
        const T m2 = fz.b * m[w].hx_z[m0] + fz.a * dHx_dz;
        m[w].hx_z[m0] = m2;
        dHx_dz = div_k(dHx_dz, fz.k) + m2;
      }
      if (py) {
        const int64_t mm = z * s1 + o1;
        const T m1 = fy.b * m[w].hz_y[mm] + fy.a * dHz_dy;
        m[w].hz_y[mm] = m1;
        dHz_dy = div_k(dHz_dy, fy.k) + m1;
        const T m2 = fy.b * m[w].hx_y[mm] + fy.a * dHx_dy;
        m[w].hx_y[mm] = m2;
        dHx_dy = div_k(dHx_dy, fy.k) + m2;
      }
      if (px) {
        const int64_t mm = z * s2 + o2;
        const T m1 = fx.b * m[w].hz_x[mm] + fx.a * dHz_dx;
        m[w].hz_x[mm] = m1;
        dHz_dx = div_k(dHz_dx, fx.k) + m1;
        const T m2 = fx.b * m[w].hy_x[mm] + fx.a * dHy_dx;
        m[w].hy_x[mm] = m2;
        dHy_dx = div_k(dHy_dx, fx.k) + m2;
      }
      cu[w][0] = dHy_dz - dHz_dy;
      cu[w][1] = dHz_dx - dHx_dz;
      cu[w][2] = dHx_dy - dHy_dx;
      p_x[w] = h_x;
      p_y[w] = h_y;
    }
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

// Sources then receivers of one step: one thread per (shot, point).
template <typename T>
__global__ void k3_points(T *__restrict__ field_src, const T *__restrict__ f_t,
                          const int64_t *__restrict__ src_i, int n_src,
                          const T *__restrict__ field_rec, T *__restrict__ r_t,
                          const int64_t *__restrict__ rec_i, int n_rec, int S, int64_t N,
                          int phase) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (phase == 0) {  // inject (duplicates within a shot accumulate in entry order)
    if (e >= S) return;
    for (int k = 0; k < n_src; ++k) {
      const int64_t c = src_i[e * n_src + k];
      if (c >= 0 && c < N) field_src[(int64_t)e * N + c] += f_t[e * n_src + k];
    }
  } else {  // record
    if (e >= S * n_rec) return;
    const int s = e / n_rec;
    const int64_t c = rec_i[e];
    r_t[e] = (c >= 0 && c < N) ? field_rec[(int64_t)s * N + c] : (T)0;
  }
}

// ---------------------------------------------------------------- adjoint
// Adjoint memories (ABI order).
enum { LEY_Z, LEZ_Y, LEZ_X, LEX_Z, LEX_Y, LEY_X, LHZ_Y, LHY_Z, LHX_Z, LHZ_X, LHY_X, LHX_Y, kNMem };
template <typename T> struct Mem12 {
  T *m[kNMem];
};

// Raw adjoint term of a cell (maxwell_3d_cuda_inst.cu:1478-1575): q (the
// signed product of coefficient and adjoint field) outside the CPML strip of
// its axis, a (b m + q) + q / kappa inside it, m the current memory adjoint.
template <typename T>
__device__ __forceinline__ T raw_term(T q, bool strip, T m, const Prof<T> &f) {
  if (!strip) return q;
  const T m_used = f.b * m + q;
  return f.a * m_used + q / f.k;
}

// Operands of one adjoint-E cell: its own coefficient and lambda_E, those of
// its y + 1 and x + 1 neighbours, and its lambda_H; loaded one cell ahead of
// the arithmetic.
template <typename T> struct OpsAE {
  T b, lx, ly, lz, by_, lzy, lxy, bx_, lzx, lyx, hx, hy, hz;
};

// Coefficient-gradient term of one stored step (maxwell_3d_cuda_inst.cu:
// 2301-2368), taken by the adjoint E launch of the next (earlier) step, which
// reads the same lambda_E: grad_ca += (lEx Ex^t + lEy Ey^t + lEz Ez^t) k and
// grad_cb likewise with curl H^t, into the per-shot buffers when several
// unbatched shots share the model.  Snapshot pointers are those of the step
// (null: that half off); `on` false: no term.
template <typename T, typename S> struct GradFold {
  const S *e[3], *c[3];
  T *gca, *gcb, *gca_shot, *gcb_shot;
  T kscale;
  bool on;
};
template <typename T, typename S>
__device__ __forceinline__ void fold_grad(const G3<T> &g, const GradFold<T, S> &gf, int64_t i,
                                          int64_t j, T lx, T ly, T lz) {
  if (!gf.on) return;
  if (gf.e[0]) {
    const T acc = lx * Snap<S, T>::dec(gf.e[0][i]) + ly * Snap<S, T>::dec(gf.e[1][i]) +
                  lz * Snap<S, T>::dec(gf.e[2][i]);
    const T v = acc * gf.kscale;
    if (g.ca_b) gf.gca[i] = gf.gca[i] + v;
    else if (g.S == 1) gf.gca[j] = gf.gca[j] + v;
    else gf.gca_shot[i] = gf.gca_shot[i] + v;
  }
  if (gf.c[0]) {
    const T acc = lx * Snap<S, T>::dec(gf.c[0][i]) + ly * Snap<S, T>::dec(gf.c[1][i]) +
                  lz * Snap<S, T>::dec(gf.c[2][i]);
    const T v = acc * gf.kscale;
    if (g.cb_b) gf.gcb[i] = gf.gcb[i] + v;
    else if (g.S == 1) gf.gcb[j] = gf.gcb[j] + v;
    else gf.gcb_shot[i] = gf.gcb_shot[i] + v;
  }
}

// Adjoint of the forward E update (maxwell_3d_cuda_inst.cu:1625-1695): next
// E-phase memory adjoints at the own cell (in their strips), lambda_H
// gathers raw terms of the own cell and of its z + 1, y + 1, x + 1
// neighbours (zero outside the update domain).  The z + 1 terms come from
// the prefetched operands of the next cell and become the own z terms of the
// next step of the march.
template <typename T, typename S>
__global__ void __launch_bounds__(256, 4)
k3_adj_e(G3<T> g, const T *__restrict__ cb, const T *__restrict__ lex,
         const T *__restrict__ ley, const T *__restrict__ lez, T *__restrict__ lhx,
         T *__restrict__ lhy, T *__restrict__ lhz, Mem12<T> cur, Mem12<T> nxt,
         GradFold<T, S> gf) {
  Col c;
  if (!column(g, c)) return;
  const int nz = g.nz, ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t sz = (int64_t)ny * nx, sy = nx;
  const int64_t base = (int64_t)c.s * g.N;
  lex += base; ley += base; lez += base; lhx += base; lhy += base; lhz += base;
  if (g.cb_b) cb += base;
  const int64_t k0 = c.s * msz0(g), k1 = c.s * msz1(g), k2 = c.s * msz2(g);
  const T *c_hy_z = cur.m[LHY_Z] + k0, *c_hx_z = cur.m[LHX_Z] + k0;
  const T *c_hz_y = cur.m[LHZ_Y] + k1, *c_hx_y = cur.m[LHX_Y] + k1;
  const T *c_hz_x = cur.m[LHZ_X] + k2, *c_hy_x = cur.m[LHY_X] + k2;
  T *n_hy_z = nxt.m[LHY_Z] + k0, *n_hx_z = nxt.m[LHX_Z] + k0;
  T *n_hz_y = nxt.m[LHZ_Y] + k1, *n_hx_y = nxt.m[LHX_Y] + k1;
  T *n_hz_x = nxt.m[LHZ_X] + k2, *n_hy_x = nxt.m[LHY_X] + k2;
  // strip state and profiles of the column and of its y + 1 / x + 1 neighbours
  auto in_y = [&](int v) { return v < g.y0 || v >= g.y1; };
  auto in_x = [&](int v) { return v < g.x0 || v >= g.x1; };
  const bool py = in_y(y), px = in_x(x);
  const bool y1ok = y + 1 < ny, x1ok = x + 1 < nx;
  const bool py1 = y1ok && in_y(y + 1), px1 = x1ok && in_x(x + 1);
  const Prof<T> fy = prof_at(g, PAY, PKY, y, py), fx = prof_at(g, PAX, PKX, x, px);
  const Prof<T> fy1 = prof_at(g, PAY, PKY, y + 1, py1), fx1 = prof_at(g, PAX, PKX, x + 1, px1);
  const int64_t s1 = (int64_t)g.eyc * nx, s2 = (int64_t)ny * g.exc;
  const int64_t o1 = (int64_t)ccoord(y, g.y0, g.yhs) * nx + x;
  const int64_t o1n = (int64_t)ccoord(y + 1, g.y0, g.yhs) * nx + x;
  const int64_t o2 = (int64_t)y * g.exc + ccoord(x, g.x0, g.xhs);
  const int64_t o2n = (int64_t)y * g.exc + ccoord(x + 1, g.x0, g.xhs);
  auto load = [&](int64_t jj) {
    OpsAE<T> o{};
    o.b = ld(cb + jj);
    o.lx = ld(lex + jj);
    o.ly = ld(ley + jj);
    o.lz = ld(lez + jj);
    if (y1ok) {
      o.by_ = ld(cb + jj + sy);
      o.lzy = ld(lez + jj + sy);
      o.lxy = ld(lex + jj + sy);
    }
    if (x1ok) {
      o.bx_ = ld(cb + jj + 1);
      o.lzx = ld(lez + jj + 1);
      o.lyx = ld(ley + jj + 1);
    }
    o.hx = lhx[jj];
    o.hy = lhy[jj];
    o.hz = lhz[jj];
    return o;
  };
  // z-axis raw terms of cell z from its coefficient and lambda_E: r_hx from
  // -cb ley with m_hx_z, r_hy from cb lex with m_hy_z
  auto raw_z = [&](int z, T b, T lx, T ly, T &r_hx, T &r_hy) {
    const T q_hx = -(b * ly), q_hy = b * lx;
    const bool pz = z < g.z0 || z >= g.z1;
    T m_hx = 0, m_hy = 0;
    Prof<T> fz{(T)0, (T)0, (T)1};
    if (pz) {
      const int64_t m = ((int64_t)ccoord(z, g.z0, g.zhs) * ny + y) * nx + x;
      m_hx = ld(c_hx_z + m);
      m_hy = ld(c_hy_z + m);
      fz = prof_at(g, PAZ, PKZ, z, true);
    }
    r_hx = raw_term(q_hx, pz, m_hx, fz);
    r_hy = raw_term(q_hy, pz, m_hy, fz);
  };
  int64_t j = ((int64_t)c.zb * ny + y) * nx + x;
  OpsAE<T> o = load(j);
  T rz_hx, rz_hy;
  raw_z(c.zb, o.b, o.lx, o.ly, rz_hx, rz_hy);
  for (int z = c.zb; z < c.ze; ++z, j += sz) {
    // next cell's operands (also the z + 1 neighbour's), zero past the last plane
    OpsAE<T> on{};
    if (z + 1 < nz) on = load(j + sz);
    const T qx = o.b * o.lx, qy = o.b * o.ly, qz = o.b * o.lz;
    fold_grad(g, gf, base + j, j, o.lx, o.ly, o.lz);
    if (z < g.z0 || z >= g.z1) {
      const int64_t m = ((int64_t)ccoord(z, g.z0, g.zhs) * ny + y) * nx + x;
      const T bz = ld(g.p[PBZ] + z);
      n_hy_z[m] = bz * ld(c_hy_z + m) + qx;
      n_hx_z[m] = bz * ld(c_hx_z + m) - qy;
    }
    T m_zy = 0, m_xy = 0, m_zx = 0, m_yx = 0;
    if (py) {
      const int64_t m = z * s1 + o1;
      m_zy = ld(c_hz_y + m);
      m_xy = ld(c_hx_y + m);
      n_hz_y[m] = fy.b * m_zy - qx;
      n_hx_y[m] = fy.b * m_xy + qz;
    }
    if (px) {
      const int64_t m = z * s2 + o2;
      m_zx = ld(c_hz_x + m);
      m_yx = ld(c_hy_x + m);
      n_hz_x[m] = fx.b * m_zx + qy;
      n_hy_x[m] = fx.b * m_yx - qz;
    }
    T rz1_hx = 0, rz1_hy = 0;
    if (z + 1 < nz) raw_z(z + 1, on.b, on.lx, on.ly, rz1_hx, rz1_hy);
    // own y / x terms
    const T ry_hx = raw_term(qz, py, m_xy, fy);   // cb lez, m_hx_y
    const T ry_hz = raw_term(-qx, py, m_zy, fy);  // -cb lex, m_hz_y
    const T rx_hy = raw_term(-qz, px, m_yx, fx);  // -cb lez, m_hy_x
    const T rx_hz = raw_term(qy, px, m_zx, fx);   // cb ley, m_hz_x
    // y + 1 and x + 1 neighbours' terms
    T ry1_hx = 0, ry1_hz = 0, rx1_hy = 0, rx1_hz = 0;
    if (y1ok) {
      T mxy = 0, mzy = 0;
      if (py1) {
        const int64_t m = z * s1 + o1n;
        mxy = ld(c_hx_y + m);
        mzy = ld(c_hz_y + m);
      }
      ry1_hx = raw_term(o.by_ * o.lzy, py1, mxy, fy1);
      ry1_hz = raw_term(-(o.by_ * o.lxy), py1, mzy, fy1);
    }
    if (x1ok) {
      T myx = 0, mzx = 0;
      if (px1) {
        const int64_t m = z * s2 + o2n;
        myx = ld(c_hy_x + m);
        mzx = ld(c_hz_x + m);
      }
      rx1_hy = raw_term(-(o.bx_ * o.lzx), px1, myx, fx1);
      rx1_hz = raw_term(o.bx_ * o.lyx, px1, mzx, fx1);
    }
    const T a1 = (rz_hx * (T)1 - rz1_hx * (T)1) * g.rdz;
    const T a2 = (ry_hx * (T)1 - ry1_hx * (T)1) * g.rdy;
    lhx[j] = o.hx + (a1 + a2);
    const T b1 = (rz_hy * (T)1 - rz1_hy * (T)1) * g.rdz;
    const T b2 = (rx_hy * (T)1 - rx1_hy * (T)1) * g.rdx;
    lhy[j] = o.hy + (b1 + b2);
    const T c1 = (ry_hz * (T)1 - ry1_hz * (T)1) * g.rdy;
    const T c2 = (rx_hz * (T)1 - rx1_hz * (T)1) * g.rdx;
    lhz[j] = o.hz + (c1 + c2);
    rz_hx = rz1_hx;
    rz_hy = rz1_hy;
    o = on;
  }
}

// Operands of one adjoint-H cell: its coefficients, lambda_H and lambda_E,
// and the coefficient and lambda_H of its y - 1 and x - 1 neighbours; loaded
// one cell ahead of the arithmetic.
template <typename T> struct OpsAH {
  T q, hx, hy, hz, a, ex, ey, ez, qy_, hzy, hxy, qx_, hzx, hyx;
};

// Adjoint of the forward H update (maxwell_3d_cuda_inst.cu:1748-1829): next
// H-phase memory adjoints at the own cell (in their strips), lambda_E gathers
// raw terms of its z - 1, y - 1, x - 1 neighbours and of the own cell (zero
// outside the update domain and on the last plane of their axis); the own
// z terms of a cell are the z - 1 terms of the next cell of the march.
template <typename T>
__global__ void __launch_bounds__(256, 3)
k3_adj_h(G3<T> g, const T *__restrict__ ca, const T *__restrict__ cq,
         const T *__restrict__ lhx, const T *__restrict__ lhy, const T *__restrict__ lhz,
         T *__restrict__ lex, T *__restrict__ ley, T *__restrict__ lez, Mem12<T> cur,
         Mem12<T> nxt) {
  Col c;
  if (!column(g, c)) return;
  const int nz = g.nz, ny = g.ny, nx = g.nx, y = c.y, x = c.x;
  const int64_t sz = (int64_t)ny * nx, sy = nx;
  const int64_t base = (int64_t)c.s * g.N;
  lhx += base; lhy += base; lhz += base; lex += base; ley += base; lez += base;
  if (g.ca_b) ca += base;
  if (g.cq_b) cq += base;
  const int64_t k0 = c.s * msz0(g), k1 = c.s * msz1(g), k2 = c.s * msz2(g);
  const T *c_ey_z = cur.m[LEY_Z] + k0, *c_ex_z = cur.m[LEX_Z] + k0;
  const T *c_ez_y = cur.m[LEZ_Y] + k1, *c_ex_y = cur.m[LEX_Y] + k1;
  const T *c_ez_x = cur.m[LEZ_X] + k2, *c_ey_x = cur.m[LEY_X] + k2;
  T *n_ey_z = nxt.m[LEY_Z] + k0, *n_ex_z = nxt.m[LEX_Z] + k0;
  T *n_ez_y = nxt.m[LEZ_Y] + k1, *n_ex_y = nxt.m[LEX_Y] + k1;
  T *n_ez_x = nxt.m[LEZ_X] + k2, *n_ey_x = nxt.m[LEY_X] + k2;
  // raw terms exist for coordinates in [1, n - 1); strips use the half-cell bounds
  auto in_y = [&](int v) { return v < g.y0 || v >= g.y1h; };
  auto in_x = [&](int v) { return v < g.x0 || v >= g.x1h; };
  const bool yok = y < ny - 1, xok = x < nx - 1;
  const bool py = yok && in_y(y), px = xok && in_x(x);
  const bool ymok = y - 1 >= 1, xmok = x - 1 >= 1;
  const bool pym = ymok && in_y(y - 1), pxm = xmok && in_x(x - 1);
  const Prof<T> fy = prof_at(g, PAYH, PKYH, y, py), fx = prof_at(g, PAXH, PKXH, x, px);
  const Prof<T> fym = prof_at(g, PAYH, PKYH, y - 1, pym);
  const Prof<T> fxm = prof_at(g, PAXH, PKXH, x - 1, pxm);
  const int64_t s1 = (int64_t)g.eyc * nx, s2 = (int64_t)ny * g.exc;
  const int64_t o1 = (int64_t)ccoord(y, g.y0, g.yhs) * nx + x;
  const int64_t o1m = (int64_t)ccoord(y - 1, g.y0, g.yhs) * nx + x;
  const int64_t o2 = (int64_t)y * g.exc + ccoord(x, g.x0, g.xhs);
  const int64_t o2m = (int64_t)y * g.exc + ccoord(x - 1, g.x0, g.xhs);
  auto load = [&](int64_t jj) {
    OpsAH<T> o{};
    o.q = ld(cq + jj);
    o.hx = ld(lhx + jj);
    o.hy = ld(lhy + jj);
    o.hz = ld(lhz + jj);
    o.a = ld(ca + jj);
    o.ex = lex[jj];
    o.ey = ley[jj];
    o.ez = lez[jj];
    if (ymok) {
      o.qy_ = ld(cq + jj - sy);
      o.hzy = ld(lhz + jj - sy);
      o.hxy = ld(lhx + jj - sy);
    }
    if (xmok) {
      o.qx_ = ld(cq + jj - 1);
      o.hzx = ld(lhz + jj - 1);
      o.hyx = ld(lhy + jj - 1);
    }
    return o;
  };
  // z-axis raw terms of cell z >= 1: r_ey from -cq lhx with m_ey_z, r_ex
  // from cq lhy with m_ex_z (zero on the last plane)
  auto raw_z = [&](int z, T q, T hx_, T hy_, T &r_ey, T &r_ex) {
    if (z >= nz - 1) {
      r_ey = r_ex = (T)0;
      return;
    }
    const T q_ey = -(q * hx_), q_ex = q * hy_;
    const bool pz = z < g.z0 || z >= g.z1h;
    T m_ey = 0, m_ex = 0;
    Prof<T> fz{(T)0, (T)0, (T)1};
    if (pz) {
      const int64_t m = ((int64_t)ccoord(z, g.z0, g.zhs) * ny + y) * nx + x;
      m_ey = ld(c_ey_z + m);
      m_ex = ld(c_ex_z + m);
      fz = prof_at(g, PAZH, PKZH, z, true);
    }
    r_ey = raw_term(q_ey, pz, m_ey, fz);
    r_ex = raw_term(q_ex, pz, m_ex, fz);
  };
  int64_t j = ((int64_t)c.zb * ny + y) * nx + x;
  T rzm_ey = 0, rzm_ex = 0;  // terms of z - 1 (zero at z - 1 = 0)
  if (c.zb - 1 >= 1)
    raw_z(c.zb - 1, ld(cq + j - sz), ld(lhx + j - sz), ld(lhy + j - sz), rzm_ey, rzm_ex);
  OpsAH<T> o = load(j);
  for (int z = c.zb; z < c.ze; ++z, j += sz) {
    OpsAH<T> on{};
    if (z + 1 < c.ze) on = load(j + sz);
    const T q = o.q, l_hx = o.hx, l_hy = o.hy, l_hz = o.hz;
    const bool zok = z < nz - 1;
    const bool pz = zok && (z < g.z0 || z >= g.z1h);
    T m_eyz = 0, m_exz = 0;
    if (pz) {
      const int64_t m = ((int64_t)ccoord(z, g.z0, g.zhs) * ny + y) * nx + x;
      const T bz = ld(g.p[PBZH] + z);
      m_eyz = ld(c_ey_z + m);
      m_exz = ld(c_ex_z + m);
      n_ey_z[m] = bz * m_eyz - q * l_hx;
      n_ex_z[m] = bz * m_exz + q * l_hy;
    }
    T m_ezy = 0, m_exy = 0, m_ezx = 0, m_eyx = 0;
    if (py) {
      const int64_t m = z * s1 + o1;
      m_ezy = ld(c_ez_y + m);
      m_exy = ld(c_ex_y + m);
      n_ez_y[m] = fy.b * m_ezy + q * l_hx;
      n_ex_y[m] = fy.b * m_exy - q * l_hz;
    }
    if (px) {
      const int64_t m = z * s2 + o2;
      m_ezx = ld(c_ez_x + m);
      m_eyx = ld(c_ey_x + m);
      n_ez_x[m] = fx.b * m_ezx - q * l_hy;
      n_ey_x[m] = fx.b * m_eyx + q * l_hz;
    }
    const T v_x = o.a * o.ex, v_y = o.a * o.ey, v_z = o.a * o.ez;
    // own terms
    T rz_ey = 0, rz_ex = 0;
    if (zok) {
      Prof<T> fz{(T)0, (T)0, (T)1};
      if (pz) fz = prof_at(g, PAZH, PKZH, z, true);
      rz_ey = raw_term(-(q * l_hx), pz, m_eyz, fz);
      rz_ex = raw_term(q * l_hy, pz, m_exz, fz);
    }
    const T rx_ey = xok ? raw_term(q * l_hz, px, m_eyx, fx) : (T)0;     // cq lhz, m_ey_x
    const T rx_ez = xok ? raw_term(-(q * l_hy), px, m_ezx, fx) : (T)0;  // -cq lhy, m_ez_x
    const T ry_ex = yok ? raw_term(-(q * l_hz), py, m_exy, fy) : (T)0;  // -cq lhz, m_ex_y
    const T ry_ez = yok ? raw_term(q * l_hx, py, m_ezy, fy) : (T)0;     // cq lhx, m_ez_y
    // y - 1 and x - 1 neighbours' terms
    T rym_ex = 0, rym_ez = 0, rxm_ey = 0, rxm_ez = 0;
    if (ymok) {
      T mexy = 0, mezy = 0;
      if (pym) {
        const int64_t m = z * s1 + o1m;
        mexy = ld(c_ex_y + m);
        mezy = ld(c_ez_y + m);
      }
      rym_ex = raw_term(-(o.qy_ * o.hzy), pym, mexy, fym);
      rym_ez = raw_term(o.qy_ * o.hxy, pym, mezy, fym);
    }
    if (xmok) {
      T meyx = 0, mezx = 0;
      if (pxm) {
        const int64_t m = z * s2 + o2m;
        meyx = ld(c_ey_x + m);
        mezx = ld(c_ez_x + m);
      }
      rxm_ey = raw_term(o.qx_ * o.hzx, pxm, meyx, fxm);
      rxm_ez = raw_term(-(o.qx_ * o.hyx), pxm, mezx, fxm);
    }
    const T e1 = (rzm_ey * (T)1 - rz_ey * (T)1) * g.rdz;
    const T e2 = (rxm_ey * (T)1 - rx_ey * (T)1) * g.rdx;
    ley[j] = v_y + (e1 + e2);
    const T f1 = (rzm_ex * (T)1 - rz_ex * (T)1) * g.rdz;
    const T f2 = (rym_ex * (T)1 - ry_ex * (T)1) * g.rdy;
    lex[j] = v_x + (f1 + f2);
    const T h1 = (rym_ez * (T)1 - ry_ez * (T)1) * g.rdy;
    const T h2 = (rxm_ez * (T)1 - rx_ez * (T)1) * g.rdx;
    lez[j] = v_z + (h1 + h2);
    rzm_ey = rz_ey;
    rzm_ex = rz_ex;
    o = on;
  }
}

#include "em3d_hi.cuh"

// Adjoint sources (receivers inject grad_r) then adjoint receivers (sources
// record grad_f), one step.
template <typename T>
__global__ void k3_adj_points(T *__restrict__ lam_rec, const T *__restrict__ gr_t,
                              const int64_t *__restrict__ rec_i, int n_rec,
                              const T *__restrict__ lam_src, T *__restrict__ gf_t,
                              const int64_t *__restrict__ src_i, int n_src, int S, int64_t N,
                              int phase) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (phase == 0) {
    if (e >= S) return;
    for (int k = 0; k < n_rec; ++k) {
      const int64_t c = rec_i[e * n_rec + k];
      if (c >= 0 && c < N) lam_rec[(int64_t)e * N + c] += gr_t[e * n_rec + k];
    }
  } else {
    if (e >= S * n_src) return;
    const int s = e / n_src;
    const int64_t c = src_i[e];
    gf_t[e] = (c >= 0 && c < N) ? lam_src[(int64_t)s * N + c] : (T)0;
  }
}

// Coefficient gradient of one stored step (maxwell_3d_cuda_inst.cu:2301-2368).
template <typename T, typename S>
__global__ void __launch_bounds__(256)
k3_coeff_grad(G3<T> g, const T *__restrict__ lex, const T *__restrict__ ley,
              const T *__restrict__ lez, const S *__restrict__ sx, const S *__restrict__ sy,
              const S *__restrict__ sz_, const S *__restrict__ cx, const S *__restrict__ cy,
              const S *__restrict__ cz, T *__restrict__ gca, T *__restrict__ gcb,
              T *__restrict__ gca_shot, T *__restrict__ gcb_shot, T kscale) {
  Cell c;
  if (!first_cell(g, c)) return;
  for (; c.z < c.zend; ++c.z) {
    set_index(c, g.ny, g.nx, g.N);
    const int64_t i = c.i;
    const T l_x = ld(lex + i), l_y = ld(ley + i), l_z = ld(lez + i);
    if (sx) {
      const T acc = l_x * Snap<S, T>::dec(sx[i]) + l_y * Snap<S, T>::dec(sy[i]) +
                    l_z * Snap<S, T>::dec(sz_[i]);
      const T v = acc * kscale;
      if (g.ca_b) gca[i] = gca[i] + v;
      else if (g.S == 1) gca[c.j] = gca[c.j] + v;
      else gca_shot[i] = gca_shot[i] + v;
    }
    if (cx) {
      const T acc = l_x * Snap<S, T>::dec(cx[i]) + l_y * Snap<S, T>::dec(cy[i]) +
                    l_z * Snap<S, T>::dec(cz[i]);
      const T v = acc * kscale;
      if (g.cb_b) gcb[i] = gcb[i] + v;
      else if (g.S == 1) gcb[c.j] = gcb[c.j] + v;
      else gcb_shot[i] = gcb_shot[i] + v;
    }
  }
}

// grad[j] += sum over shots of grad_shot[s, j] (shot order), then clear.  The
// shot loads come first and the clearing stores after them, so a thread's
// loads are all in flight together.
template <typename T>
__global__ void k3_combine(T *__restrict__ grad, T *__restrict__ shot, int S, int64_t N) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < N;
       j += (int64_t)gridDim.x * blockDim.x) {
    T sum = 0;
    for (int s = 0; s < S; ++s) sum = sum + shot[(int64_t)s * N + j];
    grad[j] = grad[j] + sum;
    for (int s = 0; s < S; ++s) shot[(int64_t)s * N + j] = (T)0;
  }
}

template <typename T>
__global__ void k3_fill(T *__restrict__ p, int64_t n, T v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// d/d(eps_r), d/d(sigma) from d/d(ca), d/d(cb) (maxwell_3d_inst.cpp:376-445).
template <typename T>
__global__ void k3_convert(const T *__restrict__ ca, const T *__restrict__ cb,
                           const T *__restrict__ gca, const T *__restrict__ gcb,
                           T *__restrict__ geps, T *__restrict__ gsig, T dt, int64_t n,
                           int64_t N, bool ca_b, bool cb_b) {
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n;
       o += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = ca_b ? o / N : 0, j = o - s * N;
    const T av = ca[ca_b ? o : j], bv = cb[cb_b ? s * N + j : j], bsq = bv * bv;
    const T ga = gca ? gca[o] : (T)0, gb = gcb ? gcb[o] : (T)0;
    const T inv_dt = (T)1 / dt;
    const T dca_de = ((T)1 - av) * bv * inv_dt, dcb_de = -bsq * inv_dt;
    const T dca_ds = -((T)0.5) * ((T)1 + av) * bv, dcb_ds = -((T)0.5) * bsq;
    if (geps) geps[o] = (ga * dca_de + gb * dcb_de) * (T)8.8541878128e-12;
    if (gsig) gsig[o] = ga * dca_ds + gb * dcb_ds;
  }
}

// ---------------------------------------------------------------- host
inline cudaStream_t stream_of(void *h) { return reinterpret_cast<cudaStream_t>(h); }

template <typename T> struct Launch3 {
  G3<T> g;
  dim3 grid, block{32, kBlockY3, 1};
  int64_t mem_size[3];  // elements of a compact memory along z, y, x
};

template <typename T>
bool make3(Launch3<T> &L, int stencil, const T *const prof[kNProf], T rdz, T rdy, T rdx, int64_t S,
           int64_t nz, int64_t ny, int64_t nx, int64_t pz0, int64_t py0, int64_t px0,
           int64_t pz1, int64_t py1, int64_t px1, bool ca_b, bool cb_b, bool cq_b,
           bool compact = true) {
  const int P = stencil / 2;
  if (S < 1 || nz < 2 * P || ny < 2 * P || nx < 2 * P || nz > (1 << 20) || ny > (1 << 20) ||
      nx > (1 << 20) || nz * ny * nx > ((int64_t)1 << 40) ||
      S * ((nz + kZRun - 1) / kZRun) > 65535) {
    set_error(kBadArgument, "3-D: unsupported shape n_shots=%lld nz=%lld ny=%lld nx=%lld",
              (long long)S, (long long)nz, (long long)ny, (long long)nx);
    return false;
  }
  for (int k = 0; k < kNProf; ++k)
    if (!prof[k]) {
      set_error(kBadArgument, "3-D: CPML profile pointer %d is null", k);
      return false;
    }
  auto bad = [](int64_t lo, int64_t hi, int64_t n) { return lo < 0 || hi < lo || hi > n; };
  if (bad(pz0, pz1, nz) || bad(py0, py1, ny) || bad(px0, px1, nx)) {
    set_error(kBadArgument, "3-D: CPML bounds outside the grid");
    return false;
  }
  G3<T> &g = L.g;
  for (int k = 0; k < kNProf; ++k) g.p[k] = prof[k];
  g.rdz = rdz; g.rdy = rdy; g.rdx = rdx;
  g.nz = (int)nz; g.ny = (int)ny; g.nx = (int)nx; g.S = (int)S;
  g.N = nz * ny * nx;
  g.z0 = (int)pz0; g.y0 = (int)py0; g.x0 = (int)px0;
  g.z1 = (int)pz1; g.y1 = (int)py1; g.x1 = (int)px1;
  g.z1h = pz1 > pz0 ? (int)pz1 - 1 : (int)pz0;
  g.y1h = py1 > py0 ? (int)py1 - 1 : (int)py0;
  g.x1h = px1 > px0 ? (int)px1 - 1 : (int)px0;
  g.zhs = (int)(compact ? std::max(pz0, pz1 - 1) : pz0);
  g.yhs = (int)(compact ? std::max(py0, py1 - 1) : py0);
  g.xhs = (int)(compact ? std::max(px0, px1 - 1) : px0);
  g.ezc = (int)pz0 + g.nz - g.zhs;
  g.eyc = (int)py0 + g.ny - g.yhs;
  g.exc = (int)px0 + g.nx - g.xhs;
  g.P = P;
  g.ca_b = ca_b; g.cb_b = cb_b; g.cq_b = cq_b;
  L.grid = dim3((unsigned)((nx + 31) / 32), (unsigned)((ny + kBlockY3 - 1) / kBlockY3),
                (unsigned)(S * ((nz + kZRun - 1) / kZRun)));
  L.mem_size[0] = S * g.ezc * ny * nx;
  L.mem_size[1] = S * nz * g.eyc * nx;
  L.mem_size[2] = S * nz * ny * g.exc;
  return true;
}

template <typename T> T *field_of(T *ex, T *ey, T *ez, int64_t comp) {
  return comp == 0 ? ex : comp == 2 ? ez : ey;
}

template <typename T>
bool common_checks(const char *what, int64_t n_src, const T *f, int64_t n_rec, const T *r,
                   int64_t src_c, int64_t rec_c, int64_t exec_backend) {
  if (n_src > 0 && !f) {
    set_error(kBadArgument, "%s: sources without amplitudes", what);
    return false;
  }
  if (n_rec > 0 && !r) {
    set_error(kBadArgument, "%s: receivers without output", what);
    return false;
  }
  if (src_c < 0 || src_c > 2 || rec_c < 0 || rec_c > 2) {
    set_error(kBadArgument, "%s: component must be 0 (x), 1 (y) or 2 (z)", what);
    return false;
  }
  if (exec_backend != 0) {
    set_error(kBadArgument, "%s: execution_backend %lld is not built (0 only)", what,
              (long long)exec_backend);
    return false;
  }
  return true;
}

template <typename T, typename S, int ST>
void launch_fwd_step(const Launch3<T> &L, cudaStream_t st, const T *ca, const T *cb,
                     const T *cq, T *F[6], T *M[12], S *const snap[6], const T *f_t,
                     const int64_t *src_i, int64_t n_src, int64_t src_c, T *r_t,
                     const int64_t *rec_i, int64_t n_rec, int64_t rec_c,
                     ProfileScope *prof = nullptr, bool smp = false) {
  if (smp) prof->begin(kK3FwdH);
  if constexpr (ST == 2)
    k3_fwd_h<T><<<L.grid, L.block, 0, st>>>(L.g, cq, F[0], F[1], F[2], F[3], F[4], F[5], M[6],
                                            M[7], M[8], M[9], M[10], M[11]);
  else
    k3p_fwd_h<T, ST / 2><<<L.grid, L.block, 0, st>>>(L.g, cq, F[0], F[1], F[2], F[3], F[4], F[5],
                                                     M[6], M[7], M[8], M[9], M[10], M[11]);
  if (smp) prof->end(kK3FwdH);
  if (smp) prof->begin(kK3FwdE);
  if constexpr (ST == 2)
    k3_fwd_e<T, S><<<L.grid, L.block, 0, st>>>(L.g, ca, cb, F[0], F[1], F[2], F[3], F[4], F[5],
                                               M[0], M[1], M[2], M[3], M[4], M[5], snap[0],
                                               snap[1], snap[2], snap[3], snap[4], snap[5]);
  else
    k3p_fwd_e<T, S, ST / 2><<<L.grid, L.block, 0, st>>>(
        L.g, ca, cb, F[0], F[1], F[2], F[3], F[4], F[5],
        BornMem<T>{M[0], M[1], M[2], M[3], M[4], M[5]}, snap[0], snap[1], snap[2], snap[3],
        snap[4], snap[5]);
  if (smp) prof->end(kK3FwdE);
  int n = 2;
  const int S_ = L.g.S;
  if (n_src > 0 && f_t && src_i) {
    k3_points<T><<<(S_ + 127) / 128, 128, 0, st>>>(field_of(F[0], F[1], F[2], src_c), f_t, src_i,
                                                   (int)n_src, nullptr, nullptr, nullptr, 0, S_,
                                                   L.g.N, 0);
    ++n;
  }
  if (n_rec > 0 && r_t && rec_i) {
    const int tot = S_ * (int)n_rec;
    k3_points<T><<<(tot + 127) / 128, 128, 0, st>>>(nullptr, nullptr, nullptr, 0,
                                                    field_of(F[0], F[1], F[2], rec_c), r_t,
                                                    rec_i, (int)n_rec, S_, L.g.N, 1);
    ++n;
  }
  count_launches(n);
}

template <typename T, int ST>
void em3d_forward(TIDE_3D_FORWARD_ARGS(T)) {
  (void)dt; (void)step_ratio; (void)n_threads; (void)n_poles;
  (void)debye_a; (void)debye_b; (void)debye_cp; (void)pol_ex; (void)pol_ey; (void)pol_ez;
  (void)ex_prev; (void)ey_prev; (void)ez_prev;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0, "3-D forward: nt must be >= 0");
  TB_REQUIRE(!has_dispersion, "3-D forward: Debye dispersion is not built in this library");
  TB_REQUIRE(ca && cb && cq && ex && ey && ez && hx && hy && hz,
             "3-D forward: a field or coefficient pointer is null");
  T *M[12] = {m_hz_y, m_hy_z, m_hx_z, m_hz_x, m_hy_x, m_hx_y,
              m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x};
  for (T *m : M) TB_REQUIRE(m != nullptr, "3-D forward: a CPML memory pointer is null");
  if (!common_checks("3-D forward", n_sources_per_shot, f, n_receivers_per_shot, r,
                     source_component, receiver_component, execution_backend))
    return;
  const T *prof[kNProf] = {az, bz, azh, bzh, ay, by, ayh, byh, ax, bx, axh, bxh,
                           kz, kzh, ky, kyh, kx, kxh};
  Launch3<T> L;
  if (!make3(L, ST, prof, rdz, rdy, rdx, n_shots, nz, ny, nx, pml_z0, pml_y0, pml_x0, pml_z1,
             pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  cudaStream_t st = stream_of(compute_stream);
  T *F[6] = {ex, ey, ez, hx, hy, hz};
  T *const none[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  ProfileScope ps(st);
  for (int64_t t = start_t; t < start_t + nt; ++t)
    launch_fwd_step<T, T, ST>(L, st, ca, cb, cq, F, M, none, f ? f + t * fs : nullptr, sources_i,
                          n_sources_per_shot, source_component, r ? r + t * rs : nullptr,
                          receivers_i, n_receivers_per_shot, receiver_component, &ps,
                          ps.sample(t));
  TB_CUDA(cudaGetLastError());
}

template <typename T, int ST>
void em3d_forward_with_storage(TIDE_3D_FORWARD_WITH_STORAGE_ARGS(T)) {
  (void)dt; (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1, "3-D forward_with_storage: bad nt/step_ratio");
  TB_REQUIRE(ca && cb && cq && ex && ey && ez && hx && hy && hz,
             "3-D forward_with_storage: a field or coefficient pointer is null");
  T *M[12] = {m_hz_y, m_hy_z, m_hx_z, m_hz_x, m_hy_x, m_hx_y,
              m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x};
  for (T *m : M) TB_REQUIRE(m != nullptr, "3-D forward_with_storage: a CPML memory is null");
  if (!common_checks("3-D forward_with_storage", n_sources_per_shot, f, n_receivers_per_shot,
                     r, source_component, receiver_component, execution_backend))
    return;
  cudaStream_t st = stream_of(compute_stream);
  StoreRun<6> sr;
  {
    void *const s1[6] = {ex_s1, ey_s1, ez_s1, cx_s1, cy_s1, cz_s1};
    void *const s3[6] = {ex_s3, ey_s3, ez_s3, cx_s3, cy_s3, cz_s3};
    char const *const *const fn[6] = {
        (char const *const *)ex_fn, (char const *const *)ey_fn, (char const *const *)ez_fn,
        (char const *const *)cx_fn, (char const *const *)cy_fn, (char const *const *)cz_fn};
    const bool need[6] = {ca_requires_grad, ca_requires_grad, ca_requires_grad,
                          cb_requires_grad, cb_requires_grad, cb_requires_grad};
    if (!sr.init("3-D", need, storage_mode, storage_format, sizeof(T), shot_bytes_uncomp,
                 nz * ny * nx, n_shots, step_ratio, s1, s3, fn, st, stream_of(storage_stream)))
      return;
  }
  const bool bf16 = sr.bf16;
  const T *prof[kNProf] = {az, bz, azh, bzh, ay, by, ayh, byh, ax, bx, axh, bxh,
                           kz, kzh, ky, kyh, kx, kxh};
  Launch3<T> L;
  if (!make3(L, ST, prof, rdz, rdy, rdx, n_shots, nz, ny, nx, pml_z0, pml_y0, pml_x0, pml_z1,
             pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  T *F[6] = {ex, ey, ez, hx, hy, hz};
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  ProfileScope ps(st);
  for (int64_t t = start_t; t < start_t + nt; ++t) {
    const bool smp = ps.sample(t);
    char *dst[6];
    if (!sr.begin(t, dst)) return;
    const T *ft = f ? f + t * fs : nullptr;
    T *rt = r ? r + t * rs : nullptr;
    if (bf16) {
      __nv_bfloat16 *const sp[6] = {(__nv_bfloat16 *)dst[0], (__nv_bfloat16 *)dst[1],
                                    (__nv_bfloat16 *)dst[2], (__nv_bfloat16 *)dst[3],
                                    (__nv_bfloat16 *)dst[4], (__nv_bfloat16 *)dst[5]};
      launch_fwd_step<T, __nv_bfloat16, ST>(L, st, ca, cb, cq, F, M, sp, ft, sources_i,
                                        n_sources_per_shot, source_component, rt, receivers_i,
                                        n_receivers_per_shot, receiver_component, &ps, smp);
    } else {
      T *const sp[6] = {(T *)dst[0], (T *)dst[1], (T *)dst[2],
                        (T *)dst[3], (T *)dst[4], (T *)dst[5]};
      launch_fwd_step<T, T, ST>(L, st, ca, cb, cq, F, M, sp, ft, sources_i, n_sources_per_shot,
                            source_component, rt, receivers_i, n_receivers_per_shot,
                            receiver_component, &ps, smp);
    }
    if (!sr.end(t, dst)) return;
  }
  if (TB_CUDA(cudaGetLastError())) return;
  sr.finish();
}

template <typename T, int ST>
void em3d_backward(TIDE_3D_BACKWARD_ARGS(T), bool compact = true) {
  (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1, "3-D backward: bad nt/step_ratio");
  TB_REQUIRE(start_t - nt >= 0, "3-D backward: start_t - nt must be >= 0");
  TB_REQUIRE(ca && cb && cq && lambda_ex && lambda_ey && lambda_ez && lambda_hx && lambda_hy &&
                 lambda_hz && adjoint_memory_scratch,
             "3-D backward: a field, coefficient or scratch pointer is null");
  TB_REQUIRE(storage_mode >= 0 && storage_mode <= 3, "3-D: unknown storage_mode %lld",
             (long long)storage_mode);
  T *lm[12] = {m_lambda_ey_z, m_lambda_ez_y, m_lambda_ez_x, m_lambda_ex_z,
               m_lambda_ex_y, m_lambda_ey_x, m_lambda_hz_y, m_lambda_hy_z,
               m_lambda_hx_z, m_lambda_hz_x, m_lambda_hy_x, m_lambda_hx_y};
  for (T *m : lm) TB_REQUIRE(m != nullptr, "3-D backward: an adjoint CPML memory is null");
  if (!common_checks<T>("3-D backward", 0, nullptr, 0, nullptr, source_component,
                        receiver_component, execution_backend))
    return;
  const bool bf16 = storage_format == 1;
  TB_REQUIRE(!bf16 || sizeof(T) == 4, "3-D: bf16 snapshot storage requires float32 fields");
  const size_t esz = bf16 ? 2 : sizeof(T);
  const bool need_ca = ca_requires_grad && grad_ca && storage_mode != 3;
  const bool need_cb = cb_requires_grad && grad_cb && storage_mode != 3;
  void *s1[6] = {ex_s1, ey_s1, ez_s1, cx_s1, cy_s1, cz_s1};
  void *s3[6] = {ex_s3, ey_s3, ez_s3, cx_s3, cy_s3, cz_s3};
  const bool need[6] = {need_ca, need_ca, need_ca, need_cb, need_cb, need_cb};
  if (need_ca || need_cb) {
    TB_REQUIRE(shot_bytes_uncomp == nz * ny * nx * (int64_t)esz,
               "3-D: shot_bytes_uncomp=%lld does not match nz*ny*nx*elem=%lld",
               (long long)shot_bytes_uncomp, (long long)(nz * ny * nx * (int64_t)esz));
    void *const fnp[6] = {ex_fn, ey_fn, ez_fn, cx_fn, cy_fn, cz_fn};
    for (int c = 0; c < 6; ++c) {
      TB_REQUIRE(!need[c] || s1[c], "3-D backward: snapshot buffer %d missing", c);
      TB_REQUIRE(!need[c] || (storage_mode != 1 && storage_mode != 2) || s3[c],
                 "3-D backward: cpu / disk storage modes need host snapshot buffer %d", c);
      TB_REQUIRE(!need[c] || storage_mode != 2 ||
                     (fnp[c] && ((char const *const *)fnp[c])[0]),
                 "3-D backward: disk storage mode needs snapshot file names");
    }
  }
  // disk mode: one reader per snapshot kind into the pinned staging ring (s3)
  std::unique_ptr<DiskHistory> disk[6];
  EventRing staged;  // the staging slot's host-to-device copy has completed
  bool staged_used[kStoreRing] = {false, false, false};
  if ((need_ca || need_cb) && storage_mode == 2) {
    if (!staged.ok) {
      set_error(kCudaError, "3-D: event creation failed");
      return;
    }
    void *const fnp[6] = {ex_fn, ey_fn, ez_fn, cx_fn, cy_fn, cz_fn};
    for (int c = 0; c < 6; ++c)
      if (need[c]) {
        disk[c].reset(new DiskHistory(((char const *const *)fnp[c])[0], false, kStoreRing));
        if (!disk[c]->ok()) {
          set_error(kBadArgument, "3-D disk storage: %s", disk[c]->error().c_str());
          return;
        }
      }
  }
  const T *prof[kNProf] = {az, bz, azh, bzh, ay, by, ayh, byh, ax, bx, axh, bxh,
                           kz, kzh, ky, kyh, kx, kxh};
  Launch3<T> L;
  if (!make3(L, ST, prof, rdz, rdy, rdx, n_shots, nz, ny, nx, pml_z0, pml_y0, pml_x0, pml_z1,
             pml_y1, pml_x1, ca_batched, cb_batched, cq_batched, compact))
    return;
  const G3<T> &g = L.g;
  const bool shot_ca = need_ca && !ca_batched && n_shots > 1;
  const bool shot_cb = need_cb && !cb_batched && n_shots > 1;
  TB_REQUIRE(!shot_ca || grad_ca_shot, "3-D backward: grad_ca_shot needed for several shots");
  TB_REQUIRE(!shot_cb || grad_cb_shot, "3-D backward: grad_cb_shot needed for several shots");
  cudaStream_t st = stream_of(compute_stream);
  const int64_t tot = n_shots * g.N;
  const int64_t model_n = g.N;
  if (zero_grad_on_entry) {
    if (grad_f && n_sources_per_shot > 0 &&
        TB_CUDA(cudaMemsetAsync(grad_f, 0, sizeof(T) * nt * n_shots * n_sources_per_shot, st)))
      return;
    if (need_ca && TB_CUDA(cudaMemsetAsync(grad_ca, 0, sizeof(T) * (ca_batched ? tot : model_n), st)))
      return;
    if (need_cb && TB_CUDA(cudaMemsetAsync(grad_cb, 0, sizeof(T) * (cb_batched ? tot : model_n), st)))
      return;
  }
  if (shot_ca && TB_CUDA(cudaMemsetAsync(grad_ca_shot, 0, sizeof(T) * tot, st))) return;
  if (shot_cb && TB_CUDA(cudaMemsetAsync(grad_cb_shot, 0, sizeof(T) * tot, st))) return;
  // Adjoint memory ping-pong: caller arrays and the scratch (same sizes).
  Mem12<T> cur, nxt;
  {
    const int axis_of[12] = {0, 1, 2, 0, 1, 2, 1, 0, 0, 2, 2, 1};
    int64_t off = 0;
    for (int m = 0; m < 12; ++m) {
      cur.m[m] = lm[m];
      nxt.m[m] = adjoint_memory_scratch + off;
      off += L.mem_size[axis_of[m]];
    }
    if (TB_CUDA(cudaMemsetAsync(adjoint_memory_scratch, 0, sizeof(T) * off, st))) return;
  }
  T *lam_src = field_of(lambda_ex, lambda_ey, lambda_ez, source_component);
  T *lam_rec = field_of(lambda_ex, lambda_ey, lambda_ez, receiver_component);
  const size_t step_bytes = (size_t)shot_bytes_uncomp * (size_t)n_shots;
  const int S_ = (int)n_shots;
  int64_t launches = 0;
  // cpu / disk modes: stored step q comes back through device ring slot
  // q % kStoreRing, loaded two stored steps ahead of its use.  With a storage
  // stream of its own the host-to-device copies run there, overlapping the
  // adjoint kernels: `loaded` orders a slot's reader after its copy and
  // `consumed` the next copy into the slot after its reader.
  const bool host_side = (need_ca || need_cb) && (storage_mode == 1 || storage_mode == 2);
  cudaStream_t ss = stream_of(storage_stream);
  const bool pipeline = host_side && ss != nullptr && ss != st;
  std::vector<int64_t> qs;  // stored steps of this call, latest first
  if (host_side)
    for (int64_t t = start_t - 1; t >= start_t - nt; --t)
      if (t % step_ratio == 0) qs.push_back(t / step_ratio);
  EventRing loaded, consumed;
  if (pipeline) {
    if (!loaded.ok || !consumed.ok) {
      set_error(kCudaError, "3-D: event creation failed");
      return;
    }
    for (int k = 0; k < kStoreRing; ++k)
      if (TB_CUDA(cudaEventRecord(consumed.ev[k], st))) return;
  }
  auto load = [&](size_t n) -> bool {
    if (n >= qs.size()) return true;
    const int64_t q = qs[n];
    const int ring = (int)(q % kStoreRing);
    cudaStream_t ls = pipeline ? ss : st;
    if (pipeline && TB_CUDA(cudaStreamWaitEvent(ss, consumed.ev[ring], 0))) return false;
    // disk mode: the staging slot is rewritten here, so its previous copy
    // to the device must have run
    if (storage_mode == 2 && staged_used[ring] && TB_CUDA(cudaEventSynchronize(staged.ev[ring])))
      return false;
    for (int c = 0; c < 6; ++c) {
      if (!need[c]) continue;
      char *slot = (char *)s1[c] + (size_t)ring * step_bytes;
      const char *host = (const char *)s3[c] + (size_t)q * step_bytes;
      if (storage_mode == 2) {
        char *stage = (char *)s3[c] + (size_t)ring * step_bytes;
        if (!disk[c]->read(stage, step_bytes, (int64_t)(q * step_bytes))) {
          set_error(kCudaError, "3-D disk storage: %s", disk[c]->error().c_str());
          return false;
        }
        host = stage;
      }
      if (TB_CUDA(cudaMemcpyAsync(slot, host, step_bytes, cudaMemcpyHostToDevice, ls)))
        return false;
    }
    if (storage_mode == 2) {
      if (TB_CUDA(cudaEventRecord(staged.ev[ring], ls))) return false;
      staged_used[ring] = true;
    }
    return !(pipeline && TB_CUDA(cudaEventRecord(loaded.ev[ring], ss)));
  };
  size_t next_n = 0;
  for (size_t n = 0; n < 2; ++n)
    if (!load(n)) return;
  int pending_ring = 0;
  ProfileScope ps(st);
  // The coefficient-gradient term of a stored step t reads lambda_E as it
  // stands after step t's receivers, which is what the adjoint E launch of
  // step t - 1 reads: that launch takes it (`pending`), and a standalone
  // pass takes the last step's.  Same additions in the same order as a
  // separate pass.
  const char *pending[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool has_pending = false;
  auto fold_of = [&](auto tag) {
    using S = decltype(tag);
    GradFold<T, S> f{};
    f.on = has_pending;
    for (int k = 0; k < 3; ++k) {
      f.e[k] = reinterpret_cast<const S *>(pending[k]);
      f.c[k] = reinterpret_cast<const S *>(pending[3 + k]);
    }
    f.gca = grad_ca; f.gcb = grad_cb; f.gca_shot = grad_ca_shot; f.gcb_shot = grad_cb_shot;
    f.kscale = (T)step_ratio;
    return f;
  };
  auto launch_adj_e = [&](auto tag) {
    using S = decltype(tag);
    const GradFold<T, S> f = fold_of(tag);
    if constexpr (ST == 2)
      k3_adj_e<T, S><<<L.grid, L.block, 0, st>>>(g, cb, lambda_ex, lambda_ey, lambda_ez,
                                                 lambda_hx, lambda_hy, lambda_hz, cur, nxt, f);
    else
      k3p_adj_e<T, S, ST / 2><<<L.grid, L.block, 0, st>>>(g, cb, lambda_ex, lambda_ey, lambda_ez,
                                                          lambda_hx, lambda_hy, lambda_hz, cur,
                                                          nxt, f);
  };
  for (int64_t t = start_t - 1; t >= start_t - nt; --t) {
    const bool smp = ps.sample(t);
    if (smp) ps.begin(kK3AdjE);
    const bool consumes = has_pending;
    if (has_pending && bf16) launch_adj_e(__nv_bfloat16(0.f));
    else launch_adj_e(T(0));
    has_pending = false;
    if (smp) ps.end(kK3AdjE);
    if (consumes && host_side) {  // the slot just read takes the history two stored steps on
      if (pipeline && TB_CUDA(cudaEventRecord(consumed.ev[pending_ring], st))) return;
      ++next_n;
      if (!load(next_n + 1)) return;
    }
    if (smp) ps.begin(kK3AdjH);
    if constexpr (ST == 2)
      k3_adj_h<T><<<L.grid, L.block, 0, st>>>(g, ca, cq, lambda_hx, lambda_hy, lambda_hz,
                                              lambda_ex, lambda_ey, lambda_ez, cur, nxt);
    else
      k3p_adj_h<T, ST / 2><<<L.grid, L.block, 0, st>>>(g, ca, cq, lambda_hx, lambda_hy, lambda_hz,
                                                       lambda_ex, lambda_ey, lambda_ez, cur, nxt);
    if (smp) ps.end(kK3AdjH);
    launches += 2;
    if (n_receivers_per_shot > 0 && grad_r && receivers_i) {
      k3_adj_points<T><<<(S_ + 127) / 128, 128, 0, st>>>(
          lam_rec, grad_r + t * n_shots * n_receivers_per_shot, receivers_i,
          (int)n_receivers_per_shot, nullptr, nullptr, nullptr, 0, S_, g.N, 0);
      ++launches;
    }
    if (n_sources_per_shot > 0 && grad_f && sources_i) {
      const int n = S_ * (int)n_sources_per_shot;
      k3_adj_points<T><<<(n + 127) / 128, 128, 0, st>>>(
          nullptr, nullptr, nullptr, 0, lam_src, grad_f + t * n_shots * n_sources_per_shot,
          sources_i, (int)n_sources_per_shot, S_, g.N, 1);
      ++launches;
    }
    if ((need_ca || need_cb) && (t % step_ratio) == 0) {
      const int64_t q = t / step_ratio;
      const int ring = (int)(q % kStoreRing);
      // host modes: the slot loaded for q (its copy ordered before the
      // reader); device mode: the history itself
      if (pipeline && TB_CUDA(cudaStreamWaitEvent(st, loaded.ev[ring], 0))) return;
      for (int c = 0; c < 6; ++c)
        pending[c] = !need[c]    ? nullptr
                     : host_side ? (const char *)s1[c] + (size_t)ring * step_bytes
                                 : (const char *)s1[c] + (size_t)q * step_bytes;
      pending_ring = ring;
      has_pending = true;
    }
    std::swap(cur, nxt);
  }
  if (has_pending) {  // the last step's term: a pass of its own
    const T ks = (T)step_ratio;
    const char *const *src = pending;
    ps.begin(kK3Grad);
    if (bf16)
      k3_coeff_grad<T, __nv_bfloat16><<<L.grid, L.block, 0, st>>>(
          g, lambda_ex, lambda_ey, lambda_ez, (const __nv_bfloat16 *)src[0],
          (const __nv_bfloat16 *)src[1], (const __nv_bfloat16 *)src[2],
          (const __nv_bfloat16 *)src[3], (const __nv_bfloat16 *)src[4],
          (const __nv_bfloat16 *)src[5], grad_ca, grad_cb, grad_ca_shot, grad_cb_shot, ks);
    else
      k3_coeff_grad<T, T><<<L.grid, L.block, 0, st>>>(
          g, lambda_ex, lambda_ey, lambda_ez, (const T *)src[0], (const T *)src[1],
          (const T *)src[2], (const T *)src[3], (const T *)src[4], (const T *)src[5],
          grad_ca, grad_cb, grad_ca_shot, grad_cb_shot, ks);
    ps.end(kK3Grad);
    ++launches;
  }
  for (int m = 0; m < 12; ++m)
    if (cur.m[m] != lm[m]) {
      const int axis_of[12] = {0, 1, 2, 0, 1, 2, 1, 0, 0, 2, 2, 1};
      if (TB_CUDA(cudaMemcpyAsync(lm[m], cur.m[m], sizeof(T) * L.mem_size[axis_of[m]],
                                  cudaMemcpyDeviceToDevice, st)))
        return;
    }
  if (shot_ca) {
    k3_combine<T><<<592, 256, 0, st>>>(grad_ca, grad_ca_shot, S_, model_n);
    ++launches;
  }
  if (shot_cb) {
    k3_combine<T><<<592, 256, 0, st>>>(grad_cb, grad_cb_shot, S_, model_n);
    ++launches;
  }
  if ((grad_eps || grad_sigma) && (need_ca || need_cb)) {
    const int64_t n = ca_batched ? tot : model_n;
    k3_convert<T><<<592, 256, 0, st>>>(ca, cb, need_ca ? grad_ca : nullptr,
                                       need_cb ? grad_cb : nullptr, grad_eps, grad_sigma, dt, n,
                                       model_n, ca_batched, cb_batched);
    ++launches;
  }
  count_launches(launches);
  if (TB_CUDA(cudaGetLastError())) return;
  if (host_side) {
    // the caller's staging and host buffers are free once the copies ran
    if (pipeline && TB_CUDA(cudaStreamSynchronize(ss))) return;
    TB_CUDA(cudaStreamSynchronize(st));
  }
}

// Snapshot plan of born_forward_with_storage: device base pointers of the
// six background kinds (s1) and of the six scattered kinds (ds), the byte
// size of one stored step and the storage precision.
struct BornStore {
  void *s1[6];
  void *ds[6];
  size_t step_bytes;
  bool bf16;
};

template <typename S, typename T>
BornSnap<S> born_snap(const BornStore *bs, int64_t q) {
  BornSnap<S> sn{};
  if (!bs) return sn;
  const size_t off = (size_t)q * bs->step_bytes;
  auto at = [&](void *b) { return b ? reinterpret_cast<S *>(static_cast<char *>(b) + off) : nullptr; };
  for (int k = 0; k < 3; ++k) {
    sn.e[k] = at(bs->s1[k]);
    sn.c[k] = at(bs->s1[3 + k]);
    sn.de[k] = at(bs->ds[k]);
    sn.dc[k] = at(bs->ds[3 + k]);
  }
  return sn;
}

template <typename T, int ST, typename S>
void launch_born_e(const Launch3<T> &L, cudaStream_t st, const T *ca, const T *cb, const T *dca,
                   const T *dcb, T *const F[6], T *const DF[6], const BornMem<T> &mb,
                   const BornMem<T> &ms, const BornSnap<S> &sn) {
  if constexpr (ST == 2)
    k3_born_e<T, S><<<L.grid, L.block, 0, st>>>(L.g, ca, cb, dca, dcb, F[0], F[1], F[2], F[3],
                                                F[4], F[5], DF[0], DF[1], DF[2], DF[3], DF[4],
                                                DF[5], mb, ms, sn);
  else
    k3p_born_e<T, S, ST / 2><<<L.grid, L.block, 0, st>>>(L.g, ca, cb, dca, dcb, F[0], F[1], F[2],
                                                         F[3], F[4], F[5], DF[0], DF[1], DF[2],
                                                         DF[3], DF[4], DF[5], mb, ms, sn);
}

template <typename T, int ST>
void em3d_born_forward(TIDE_3D_BORN_FORWARD_ARGS(T), const BornStore *bs = nullptr) {
  (void)dt; (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1, "3-D born_forward: bad nt / step_ratio");
  TB_REQUIRE(ca && cb && cq && dca && dcb && ex && ey && ez && hx && hy && hz && dex && dey &&
                 dez && dhx && dhy && dhz,
             "3-D born_forward: a field or coefficient pointer is null");
  T *M[12] = {m_hz_y, m_hy_z, m_hx_z, m_hz_x, m_hy_x, m_hx_y,
              m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x};
  T *DM[12] = {dm_hz_y, dm_hy_z, dm_hx_z, dm_hz_x, dm_hy_x, dm_hx_y,
               dm_ey_z, dm_ez_y, dm_ez_x, dm_ex_z, dm_ex_y, dm_ey_x};
  for (int k = 0; k < 12; ++k)
    TB_REQUIRE(M[k] && DM[k], "3-D born_forward: a CPML memory pointer is null");
  TB_REQUIRE(n_sources_per_shot == 0 || (f0 && df),
             "3-D born_forward: sources without background or scattered amplitudes");
  if (!common_checks("3-D born_forward", 0, (const T *)nullptr, n_receivers_per_shot, r,
                     source_component, receiver_component, execution_backend))
    return;
  const T *prof[kNProf] = {az, bz, azh, bzh, ay, by, ayh, byh, ax, bx, axh, bxh,
                           kz, kzh, ky, kyh, kx, kxh};
  // The Born entry points take full [S, nz, ny, nx] CPML memories
  // (maxwell_3d_cuda_inst.cu:3871-3890 sets the compact flag off there).
  Launch3<T> L;
  if (!make3(L, ST, prof, rdz, rdy, rdx, n_shots, nz, ny, nx, pml_z0, pml_y0, pml_x0, pml_z1,
             pml_y1, pml_x1, ca_batched, cb_batched, cq_batched, /*compact=*/false))
    return;
  cudaStream_t st = stream_of(compute_stream);
  T *F[6] = {ex, ey, ez, hx, hy, hz}, *DF[6] = {dex, dey, dez, dhx, dhy, dhz};
  const BornMem<T> mb{M[0], M[1], M[2], M[3], M[4], M[5]};
  const BornMem<T> ms{DM[0], DM[1], DM[2], DM[3], DM[4], DM[5]};
  const int S_ = (int)n_shots;
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  int64_t launches = 0;
  for (int64_t t = start_t; t < start_t + nt; ++t) {
    T *const *fs2[2] = {F, DF};
    T *const *ms2[2] = {M, DM};
    for (int w = 0; w < 2; ++w) {
      T *const *Fw = fs2[w], *const *Mw = ms2[w];
      if constexpr (ST == 2)
        k3_fwd_h<T><<<L.grid, L.block, 0, st>>>(L.g, cq, Fw[0], Fw[1], Fw[2], Fw[3], Fw[4],
                                                Fw[5], Mw[6], Mw[7], Mw[8], Mw[9], Mw[10], Mw[11]);
      else
        k3p_fwd_h<T, ST / 2><<<L.grid, L.block, 0, st>>>(L.g, cq, Fw[0], Fw[1], Fw[2], Fw[3],
                                                         Fw[4], Fw[5], Mw[6], Mw[7], Mw[8], Mw[9],
                                                         Mw[10], Mw[11]);
    }
    const bool store = bs && t % step_ratio == 0;
    if (store && bs->bf16)
      launch_born_e<T, ST>(L, st, ca, cb, dca, dcb, F, DF, mb, ms,
                           born_snap<__nv_bfloat16, T>(bs, t / step_ratio));
    else
      launch_born_e<T, ST>(L, st, ca, cb, dca, dcb, F, DF, mb, ms,
                           born_snap<T, T>(store ? bs : nullptr, t / step_ratio));
    launches += 3;
    if (n_sources_per_shot > 0 && sources_i) {
      k3_points<T><<<(S_ + 127) / 128, 128, 0, st>>>(
          field_of(ex, ey, ez, source_component), f0 + t * fs, sources_i,
          (int)n_sources_per_shot, nullptr, nullptr, nullptr, 0, S_, L.g.N, 0);
      k3_points<T><<<(S_ + 127) / 128, 128, 0, st>>>(
          field_of(dex, dey, dez, source_component), df + t * fs, sources_i,
          (int)n_sources_per_shot, nullptr, nullptr, nullptr, 0, S_, L.g.N, 0);
      launches += 2;
    }
    if (n_receivers_per_shot > 0 && receivers_i) {
      const int tot = S_ * (int)n_receivers_per_shot;
      if (r) {
        k3_points<T><<<(tot + 127) / 128, 128, 0, st>>>(
            nullptr, nullptr, nullptr, 0, field_of(dex, dey, dez, receiver_component),
            r + t * rs, receivers_i, (int)n_receivers_per_shot, S_, L.g.N, 1);
        ++launches;
      }
      if (background_r) {
        k3_points<T><<<(tot + 127) / 128, 128, 0, st>>>(
            nullptr, nullptr, nullptr, 0, field_of(ex, ey, ez, receiver_component),
            background_r + t * rs, receivers_i, (int)n_receivers_per_shot, S_, L.g.N, 1);
        ++launches;
      }
    }
  }
  count_launches(launches);
  TB_CUDA(cudaGetLastError());
}

// ------------------------------------------- second-order Born adjoint
// The 3-D joint adjoint of the background and scattered recurrences (see the
// 2-D version in tm2d_born.cuh): lam = the scattered state's adjoint (driven
// by grad_r), eta = the background's.  Per step, with both at t+1:
// W = cb eta_E + dcb lam_E and eta_E <- ca eta_E + dca lam_E (k3_bg_prep),
// the adjoint phases of lam (cb, ca) and of eta (W as the E-phase input,
// unit ca), sources grad_f0 <- eta and grad_df <- lam, receivers grad_r ->
// lam; at stored steps grad_ca += eta.E + lam.dE, grad_cb += eta.curl +
// lam.dcurl, grad_dca += lam.E, grad_dcb += lam.curl (times k), per shot
// when several unbatched shots share the model, summed at the end.
template <typename T>
__global__ void __launch_bounds__(256)
k3_bg_prep(G3<T> g, const T *__restrict__ ca, const T *__restrict__ cb,
           const T *__restrict__ dca, const T *__restrict__ dcb, const T *__restrict__ lex,
           const T *__restrict__ ley, const T *__restrict__ lez, T *__restrict__ eex,
           T *__restrict__ eey, T *__restrict__ eez, T *__restrict__ w0, T *__restrict__ w1,
           T *__restrict__ w2) {
  Col c;
  if (!column(g, c)) return;
  const int64_t base = (int64_t)c.s * g.N;
  const T *L[3] = {lex + base, ley + base, lez + base};
  T *E[3] = {eex + base, eey + base, eez + base}, *W[3] = {w0 + base, w1 + base, w2 + base};
  if (g.ca_b) { ca += base; dca += base; }
  if (g.cb_b) { cb += base; dcb += base; }
  for (int z = c.zb; z < c.ze; ++z) {
    const int64_t j = ((int64_t)z * g.ny + c.y) * g.nx + c.x;
    const T a = ld(ca + j), da = ld(dca + j), b = ld(cb + j), db = ld(dcb + j);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T l = L[k][j], e = E[k][j];
      W[k][j] = b * e + db * l;
      E[k][j] = a * e + da * l;
    }
  }
}

template <typename T, int ST>
void em3d_born_backward_bggrad(TIDE_3D_BORN_BACKWARD_BGGRAD_ARGS(T)) {
  (void)f0; (void)df; (void)n_threads; (void)storage_stream; (void)dt;
  (void)ex_s3; (void)ex_fn; (void)ey_s3; (void)ey_fn; (void)ez_s3; (void)ez_fn;
  (void)cx_s3; (void)cx_fn; (void)cy_s3; (void)cy_fn; (void)cz_s3; (void)cz_fn;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1 && start_t - nt >= 0,
             "3-D born_backward_bggrad: bad nt/step_ratio/start_t");
  TB_REQUIRE(storage_mode == 0, "3-D born_backward_bggrad: device storage mode only");
  T *lam[6] = {lambda_ex, lambda_ey, lambda_ez, lambda_hx, lambda_hy, lambda_hz};
  T *eta[6] = {eta_ex, eta_ey, eta_ez, eta_hx, eta_hy, eta_hz};
  T *lm[12] = {m_lambda_ey_z, m_lambda_ez_y, m_lambda_ez_x, m_lambda_ex_z,
               m_lambda_ex_y, m_lambda_ey_x, m_lambda_hz_y, m_lambda_hy_z,
               m_lambda_hx_z, m_lambda_hz_x, m_lambda_hy_x, m_lambda_hx_y};
  T *em[12] = {m_eta_ey_z, m_eta_ez_y, m_eta_ez_x, m_eta_ex_z, m_eta_ex_y, m_eta_ey_x,
               m_eta_hz_y, m_eta_hy_z, m_eta_hx_z, m_eta_hz_x, m_eta_hy_x, m_eta_hx_y};
  for (int k = 0; k < 6; ++k)
    TB_REQUIRE(lam[k] && eta[k], "3-D born_backward_bggrad: an adjoint field is null");
  for (int k = 0; k < 12; ++k)
    TB_REQUIRE(lm[k] && em[k], "3-D born_backward_bggrad: an adjoint memory is null");
  TB_REQUIRE(ca && cb && cq && dca && dcb && adjoint_memory_scratch && eta_source_ex &&
                 eta_source_ey && eta_source_ez,
             "3-D born_backward_bggrad: a coefficient, scratch or work pointer is null");
  if (!common_checks<T>("3-D born_backward_bggrad", 0, nullptr, 0, nullptr, source_component,
                        receiver_component, execution_backend))
    return;
  const bool bf16 = storage_format == 1;
  TB_REQUIRE(!bf16 || sizeof(T) == 4, "3-D: bf16 snapshot storage requires float32 fields");
  const size_t esz = bf16 ? 2 : sizeof(T);
  TB_REQUIRE(shot_bytes_uncomp == nz * ny * nx * (int64_t)esz,
             "3-D born_backward_bggrad: shot_bytes_uncomp does not match nz*ny*nx*elem");
  const bool need[4] = {ca_requires_grad && grad_ca, cb_requires_grad && grad_cb,
                        dca_requires_grad && grad_dca, dcb_requires_grad && grad_dcb};
  void *bg_st[6] = {ex_s1, ey_s1, ez_s1, cx_s1, cy_s1, cz_s1};
  void *sc_st[6] = {dex_store, dey_store, dez_store, dcurl_x_store, dcurl_y_store,
                    dcurl_z_store};
  for (int k = 0; k < 6; ++k) {
    const bool e = k < 3;
    TB_REQUIRE(!((e ? need[0] || need[2] : need[1] || need[3]) && !bg_st[k]),
               "3-D born_backward_bggrad: background history %d missing", k);
    TB_REQUIRE(!((e ? need[0] : need[1]) && !sc_st[k]),
               "3-D born_backward_bggrad: scattered history %d missing", k);
  }
  const T *prof[kNProf] = {az, bz, azh, bzh, ay, by, ayh, byh, ax, bx, axh, bxh,
                           kz, kzh, ky, kyh, kx, kxh};
  Launch3<T> L;
  if (!make3(L, ST, prof, rdz, rdy, rdx, n_shots, nz, ny, nx, pml_z0, pml_y0, pml_x0, pml_z1,
             pml_y1, pml_x1, ca_batched, cb_batched, cq_batched, /*compact=*/false))
    return;
  const G3<T> &g = L.g;
  cudaStream_t st = stream_of(compute_stream);
  const int64_t tot = n_shots * g.N;
  const size_t tb = sizeof(T) * (size_t)tot;
  for (int k = 0; k < 6; ++k)
    if (TB_CUDA(cudaMemsetAsync(lam[k], 0, tb, st)) || TB_CUDA(cudaMemsetAsync(eta[k], 0, tb, st)))
      return;
  for (int k = 0; k < 12; ++k)
    if (TB_CUDA(cudaMemsetAsync(lm[k], 0, tb, st)) || TB_CUDA(cudaMemsetAsync(em[k], 0, tb, st)))
      return;
  if (TB_CUDA(cudaMemsetAsync(adjoint_memory_scratch, 0, 24 * tb, st))) return;
  T *wf[3] = {eta_source_ex, eta_source_ey, eta_source_ez};
  for (int k = 0; k < 3; ++k)
    if (TB_CUDA(cudaMemsetAsync(wf[k], 0, tb, st))) return;
  const bool shots = n_shots > 1;
  T *gout[4] = {grad_ca, grad_cb, grad_dca, grad_dcb};
  T *gshot[4] = {grad_ca_shot, grad_cb_shot, grad_dca_shot, grad_dcb_shot};
  const bool batched_of[4] = {ca_batched, cb_batched, ca_batched, cb_batched};
  for (int q = 0; q < 4; ++q)
    if (need[q] && shots && !batched_of[q]) {
      TB_REQUIRE(gshot[q], "3-D born_backward_bggrad: per-shot gradient buffer %d missing", q);
      if (TB_CUDA(cudaMemsetAsync(gshot[q], 0, tb, st))) return;
    }
  T *ones = nullptr;
  if (TB_CUDA(pool_malloc((void **)&ones, tb, st))) return;
  k3_fill<T><<<592, 256, 0, st>>>(ones, tot, (T)1);
  Mem12<T> lc, ln, ec, en;
  for (int m = 0; m < 12; ++m) {
    lc.m[m] = lm[m];
    ln.m[m] = adjoint_memory_scratch + m * tot;
    ec.m[m] = em[m];
    en.m[m] = adjoint_memory_scratch + (12 + m) * tot;
  }
  const GradFold<T, T> off{};
  auto adj_e = [&](const T *b, T *const F[6], Mem12<T> c, Mem12<T> n) {
    if constexpr (ST == 2)
      k3_adj_e<T, T><<<L.grid, L.block, 0, st>>>(g, b, F[0], F[1], F[2], F[3], F[4], F[5], c, n,
                                                 off);
    else
      k3p_adj_e<T, T, ST / 2><<<L.grid, L.block, 0, st>>>(g, b, F[0], F[1], F[2], F[3], F[4],
                                                          F[5], c, n, off);
  };
  auto adj_h = [&](const T *a, T *const F[6], Mem12<T> c, Mem12<T> n) {
    if constexpr (ST == 2)
      k3_adj_h<T><<<L.grid, L.block, 0, st>>>(g, a, cq, F[3], F[4], F[5], F[0], F[1], F[2], c, n);
    else
      k3p_adj_h<T, ST / 2><<<L.grid, L.block, 0, st>>>(g, a, cq, F[3], F[4], F[5], F[0], F[1],
                                                       F[2], c, n);
  };
  auto image = [&](T *const F[6], void *const s6[6], size_t off_b, T *ga, T *gb, T *gas,
                   T *gbs, bool na, bool nb) {
    if (!na && !nb) return;
    const char *p[6];
    for (int k = 0; k < 6; ++k) p[k] = (k < 3 ? na : nb) ? (const char *)s6[k] + off_b : nullptr;
    if (bf16)
      k3_coeff_grad<T, __nv_bfloat16><<<L.grid, L.block, 0, st>>>(
          g, F[0], F[1], F[2], (const __nv_bfloat16 *)p[0], (const __nv_bfloat16 *)p[1],
          (const __nv_bfloat16 *)p[2], (const __nv_bfloat16 *)p[3], (const __nv_bfloat16 *)p[4],
          (const __nv_bfloat16 *)p[5], ga, gb, gas, gbs, (T)step_ratio);
    else
      k3_coeff_grad<T, T><<<L.grid, L.block, 0, st>>>(
          g, F[0], F[1], F[2], (const T *)p[0], (const T *)p[1], (const T *)p[2],
          (const T *)p[3], (const T *)p[4], (const T *)p[5], ga, gb, gas, gbs, (T)step_ratio);
  };
  T *W6[6] = {wf[0], wf[1], wf[2], eta[3], eta[4], eta[5]};
  const int S_ = (int)n_shots;
  const size_t step_bytes = (size_t)shot_bytes_uncomp * (size_t)n_shots;
  int64_t launches = 1;
  for (int64_t t = start_t - 1; t >= start_t - nt; --t) {
    k3_bg_prep<T><<<L.grid, L.block, 0, st>>>(g, ca, cb, dca, dcb, lam[0], lam[1], lam[2], eta[0],
                                              eta[1], eta[2], wf[0], wf[1], wf[2]);
    adj_e(cb, lam, lc, ln);
    adj_e(ones, W6, ec, en);
    adj_h(ones, eta, ec, en);
    if (n_sources_per_shot > 0 && grad_f0 && sources_i) {
      const int n = S_ * (int)n_sources_per_shot;
      k3_adj_points<T><<<(n + 127) / 128, 128, 0, st>>>(
          nullptr, nullptr, nullptr, 0, field_of(eta[0], eta[1], eta[2], source_component),
          grad_f0 + t * n_shots * n_sources_per_shot, sources_i, (int)n_sources_per_shot, S_,
          g.N, 1);
      ++launches;
    }
    adj_h(ca, lam, lc, ln);
    if (n_receivers_per_shot > 0 && grad_r && receivers_i) {
      k3_adj_points<T><<<(S_ + 127) / 128, 128, 0, st>>>(
          field_of(lam[0], lam[1], lam[2], receiver_component),
          grad_r + t * n_shots * n_receivers_per_shot, receivers_i, (int)n_receivers_per_shot,
          nullptr, nullptr, nullptr, 0, S_, g.N, 0);
      ++launches;
    }
    if (n_sources_per_shot > 0 && grad_df && sources_i) {
      const int n = S_ * (int)n_sources_per_shot;
      k3_adj_points<T><<<(n + 127) / 128, 128, 0, st>>>(
          nullptr, nullptr, nullptr, 0, field_of(lam[0], lam[1], lam[2], source_component),
          grad_df + t * n_shots * n_sources_per_shot, sources_i, (int)n_sources_per_shot, S_,
          g.N, 1);
      ++launches;
    }
    std::swap(lc, ln);
    std::swap(ec, en);
    launches += 5;
    if (t % step_ratio == 0) {
      const size_t ob = (size_t)(t / step_ratio) * step_bytes;
      image(eta, bg_st, ob, gout[0], gout[1], gshot[0], gshot[1], need[0], need[1]);
      image(lam, sc_st, ob, gout[0], gout[1], gshot[0], gshot[1], need[0], need[1]);
      image(lam, bg_st, ob, gout[2], gout[3], gshot[2], gshot[3], need[2], need[3]);
      launches += 3;
    }
  }
  for (int m = 0; m < 12; ++m) {
    if (lc.m[m] != lm[m] && TB_CUDA(cudaMemcpyAsync(lm[m], lc.m[m], tb, cudaMemcpyDeviceToDevice,
                                                    st)))
      return;
    if (ec.m[m] != em[m] && TB_CUDA(cudaMemcpyAsync(em[m], ec.m[m], tb, cudaMemcpyDeviceToDevice,
                                                    st)))
      return;
  }
  for (int q = 0; q < 4; ++q)
    if (need[q] && shots && !batched_of[q]) {
      k3_combine<T><<<592, 256, 0, st>>>(gout[q], gshot[q], S_, g.N);
      ++launches;
    }
  count_launches(launches);
  TB_CUDA(cudaFreeAsync(ones, st));
  TB_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace tb

#define TB3_DEFINE(S, T)                                                                   \
  extern "C" void maxwell_3d_##S##_##T##_forward_cuda(TIDE_3D_FORWARD_ARGS(T)) {           \
    tb::em3d_forward<T, S>(                                                                   \
        ca, cb, cq, f, ex, ey, ez, hx, hy, hz, m_hz_y, m_hy_z, m_hx_z, m_hz_x, m_hy_x,     \
        m_hx_y, m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x, debye_a, debye_b,          \
        debye_cp, pol_ex, pol_ey, pol_ez, ex_prev, ey_prev, ez_prev, r, n_poles, az, bz,   \
        azh, bzh, ay, by, ayh, byh, ax, bx, axh, bxh, kz, kzh, ky, kyh, kx, kxh,           \
        sources_i, receivers_i, rdz, rdy, rdx, dt, nt, n_shots, nz, ny, nx,                \
        n_sources_per_shot, n_receivers_per_shot, step_ratio, has_dispersion, ca_batched,  \
        cb_batched, cq_batched, start_t, pml_z0, pml_y0, pml_x0, pml_z1, pml_y1, pml_x1,   \
        source_component, receiver_component, n_threads, device, execution_backend,        \
        compute_stream);                                                                   \
  }                                                                                        \
  extern "C" void maxwell_3d_##S##_##T##_forward_with_storage_cuda(                        \
      TIDE_3D_FORWARD_WITH_STORAGE_ARGS(T)) {                                              \
    tb::em3d_forward_with_storage<T, S>(                                                      \
        ca, cb, cq, f, ex, ey, ez, hx, hy, hz, m_hz_y, m_hy_z, m_hx_z, m_hz_x, m_hy_x,     \
        m_hx_y, m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x, r, ex_s1, ex_s3, ex_fn,    \
        ey_s1, ey_s3, ey_fn, ez_s1, ez_s3, ez_fn, cx_s1, cx_s3, cx_fn, cy_s1, cy_s3,       \
        cy_fn, cz_s1, cz_s3, cz_fn, az, bz, azh, bzh, ay, by, ayh, byh, ax, bx, axh, bxh,  \
        kz, kzh, ky, kyh, kx, kxh, sources_i, receivers_i, rdz, rdy, rdx, dt, nt, n_shots, \
        nz, ny, nx, n_sources_per_shot, n_receivers_per_shot, step_ratio, storage_mode,    \
        storage_format, shot_bytes_uncomp, ca_requires_grad, cb_requires_grad, ca_batched, \
        cb_batched, cq_batched, start_t, pml_z0, pml_y0, pml_x0, pml_z1, pml_y1, pml_x1,   \
        source_component, receiver_component, n_threads, device, execution_backend,        \
        compute_stream, storage_stream);                                                   \
  }                                                                                        \
  extern "C" void maxwell_3d_##S##_##T##_backward_cuda(TIDE_3D_BACKWARD_ARGS(T)) {         \
    tb::em3d_backward<T, S>(                                                                  \
        ca, cb, cq, grad_r, lambda_ex, lambda_ey, lambda_ez, lambda_hx, lambda_hy,         \
        lambda_hz, m_lambda_ey_z, m_lambda_ez_y, m_lambda_ez_x, m_lambda_ex_z,             \
        m_lambda_ex_y, m_lambda_ey_x, m_lambda_hz_y, m_lambda_hy_z, m_lambda_hx_z,         \
        m_lambda_hz_x, m_lambda_hy_x, m_lambda_hx_y, adjoint_memory_scratch, ex_s1, ex_s3, \
        ex_fn, ey_s1, ey_s3, ey_fn, ez_s1, ez_s3, ez_fn, cx_s1, cx_s3, cx_fn, cy_s1,       \
        cy_s3, cy_fn, cz_s1, cz_s3, cz_fn, grad_f, grad_ca, grad_cb, grad_eps, grad_sigma, \
        grad_ca_shot, grad_cb_shot, zero_grad_on_entry, az, bz, azh, bzh, ay, by, ayh,     \
        byh, ax, bx, axh, bxh, kz, kzh, ky, kyh, kx, kxh, sources_i, receivers_i, rdz,     \
        rdy, rdx, dt, nt, n_shots, nz, ny, nx, n_sources_per_shot, n_receivers_per_shot,   \
        step_ratio, storage_mode, storage_format, shot_bytes_uncomp, ca_requires_grad,     \
        cb_requires_grad, ca_batched, cb_batched, cq_batched, start_t, pml_z0, pml_y0,     \
        pml_x0, pml_z1, pml_y1, pml_x1, source_component, receiver_component, n_threads,   \
        device, execution_backend, compute_stream, storage_stream);                        \
  }

TB3_DEFINE(2, float)
TB3_DEFINE(2, double)
TB3_DEFINE(4, float)
TB3_DEFINE(4, double)
TB3_DEFINE(6, float)
TB3_DEFINE(6, double)
TB3_DEFINE(8, float)
TB3_DEFINE(8, double)

#define TB3_BORN_DEFINE(S, T)                                                              \
  extern "C" void maxwell_3d_##S##_##T##_born_forward_cuda(TIDE_3D_BORN_FORWARD_ARGS(T)) { \
    tb::em3d_born_forward<T, S>(                                                              \
        ca, cb, cq, dca, dcb, f0, df, ex, ey, ez, hx, hy, hz, m_hz_y, m_hy_z, m_hx_z,      \
        m_hz_x, m_hy_x, m_hx_y, m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x, dex, dey,  \
        dez, dhx, dhy, dhz, dm_hz_y, dm_hy_z, dm_hx_z, dm_hz_x, dm_hy_x, dm_hx_y, dm_ey_z, \
        dm_ez_y, dm_ez_x, dm_ex_z, dm_ex_y, dm_ey_x, r, background_r, az, bz, azh, bzh,   \
        ay, by, ayh, byh, ax, bx, axh, bxh, kz, kzh, ky, kyh, kx, kxh, sources_i,          \
        receivers_i, rdz, rdy, rdx, dt, nt, n_shots, nz, ny, nx, n_sources_per_shot,       \
        n_receivers_per_shot, step_ratio, ca_batched, cb_batched, cq_batched, start_t,     \
        pml_z0, pml_y0, pml_x0, pml_z1, pml_y1, pml_x1, source_component,                 \
        receiver_component, n_threads, device, execution_backend, compute_stream);        \
  }

#define TB3_BORN_STORE_DEFINE(S, T)                                                          \
  extern "C" void maxwell_3d_##S##_##T##_born_forward_with_storage_cuda(                   \
      TIDE_3D_BORN_FORWARD_WITH_STORAGE_ARGS(T)) {                                         \
    (void)ex_s3; (void)ex_fn; (void)ey_s3; (void)ey_fn; (void)ez_s3; (void)ez_fn;          \
    (void)cx_s3; (void)cx_fn; (void)cy_s3; (void)cy_fn; (void)cz_s3; (void)cz_fn;          \
    (void)storage_stream;                                                                  \
    tb::BornStore bs{};                                                                    \
    const size_t esz = storage_format == 1 ? 2 : sizeof(T);                                \
    /* the reference stores in device mode only, at one snapshot per shot */               \
    const bool direct = storage_mode == 0 && shot_bytes_uncomp == nz * ny * nx * (int64_t)esz; \
    if (storage_format == 1 && sizeof(T) != 4) {                                           \
      tb::set_error(tb::kBadArgument, "3-D born: bf16 snapshots need float32 fields");    \
      return;                                                                              \
    }                                                                                      \
    if (direct) {                                                                          \
      void *s1[6] = {ex_s1, ey_s1, ez_s1, cx_s1, cy_s1, cz_s1};                            \
      void *ds[6] = {dex_store, dey_store, dez_store, dcurl_x_store, dcurl_y_store,        \
                     dcurl_z_store};                                                       \
      for (int k = 0; k < 6; ++k) {                                                        \
        const bool need = k < 3 ? ca_requires_grad : cb_requires_grad;                    \
        bs.s1[k] = need ? s1[k] : nullptr;                                                 \
        bs.ds[k] = ds[k];                                                                  \
      }                                                                                    \
      for (int k = 0; k < 6; k += 3) {                                                     \
        if (!bs.s1[k] || !bs.s1[k + 1] || !bs.s1[k + 2]) bs.s1[k] = bs.s1[k + 1] =        \
            bs.s1[k + 2] = nullptr;                                                        \
        if (!bs.ds[k] || !bs.ds[k + 1] || !bs.ds[k + 2]) bs.ds[k] = bs.ds[k + 1] =        \
            bs.ds[k + 2] = nullptr;                                                        \
      }                                                                                    \
      bs.step_bytes = (size_t)shot_bytes_uncomp * (size_t)n_shots;                         \
      bs.bf16 = storage_format == 1;                                                       \
    }                                                                                      \
    tb::em3d_born_forward<T, S>(                                                           \
        ca, cb, cq, dca, dcb, f0, df, ex, ey, ez, hx, hy, hz, m_hz_y, m_hy_z, m_hx_z,      \
        m_hz_x, m_hy_x, m_hx_y, m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x, dex, dey,  \
        dez, dhx, dhy, dhz, dm_hz_y, dm_hy_z, dm_hx_z, dm_hz_x, dm_hy_x, dm_hx_y, dm_ey_z, \
        dm_ez_y, dm_ez_x, dm_ex_z, dm_ex_y, dm_ey_x, r, background_r, az, bz, azh, bzh,   \
        ay, by, ayh, byh, ax, bx, axh, bxh, kz, kzh, ky, kyh, kx, kxh, sources_i,          \
        receivers_i, rdz, rdy, rdx, dt, nt, n_shots, nz, ny, nx, n_sources_per_shot,       \
        n_receivers_per_shot, step_ratio, ca_batched, cb_batched, cq_batched, start_t,     \
        pml_z0, pml_y0, pml_x0, pml_z1, pml_y1, pml_x1, source_component,                 \
        receiver_component, n_threads, device, execution_backend, compute_stream,         \
        direct ? &bs : nullptr);                                                           \
  }                                                                                        \
  extern "C" void maxwell_3d_##S##_##T##_born_backward_cuda(TIDE_3D_BORN_BACKWARD_ARGS(T)) { \
    tb::em3d_backward<T, S>(                                                               \
        ca, cb, cq, grad_r, lambda_ex, lambda_ey, lambda_ez, lambda_hx, lambda_hy,         \
        lambda_hz, m_lambda_ey_z, m_lambda_ez_y, m_lambda_ez_x, m_lambda_ex_z,             \
        m_lambda_ex_y, m_lambda_ey_x, m_lambda_hz_y, m_lambda_hy_z, m_lambda_hx_z,         \
        m_lambda_hz_x, m_lambda_hy_x, m_lambda_hx_y, adjoint_memory_scratch, ex_s1, ex_s3, \
        ex_fn, ey_s1, ey_s3, ey_fn, ez_s1, ez_s3, ez_fn, cx_s1, cx_s3, cx_fn, cy_s1,       \
        cy_s3, cy_fn, cz_s1, cz_s3, cz_fn, grad_f, grad_ca, grad_cb, nullptr, nullptr,     \
        grad_ca_shot, grad_cb_shot, /*zero_grad_on_entry=*/true, az, bz, azh, bzh, ay, by, \
        ayh, byh, ax, bx, axh, bxh, kz, kzh, ky, kyh, kx, kxh, sources_i, receivers_i,     \
        rdz, rdy, rdx, dt, nt, n_shots, nz, ny, nx, n_sources_per_shot,                    \
        n_receivers_per_shot, step_ratio, storage_mode, storage_format, shot_bytes_uncomp, \
        ca_requires_grad, cb_requires_grad, ca_batched, cb_batched, cq_batched, start_t,   \
        pml_z0, pml_y0, pml_x0, pml_z1, pml_y1, pml_x1, source_component,                 \
        receiver_component, n_threads, device, execution_backend, compute_stream,         \
        storage_stream, /*compact=*/false);                                               \
  }

#define TB3_BGGRAD_DEFINE(S, T)                                                            \
  extern "C" void maxwell_3d_##S##_##T##_born_backward_bggrad_cuda(                        \
      TIDE_3D_BORN_BACKWARD_BGGRAD_ARGS(T)) {                                              \
    tb::em3d_born_backward_bggrad<T, S>(                                                   \
        ca, cb, cq, dca, dcb, f0, df, grad_r, lambda_ex, lambda_ey, lambda_ez, lambda_hx,  \
        lambda_hy, lambda_hz, m_lambda_ey_z, m_lambda_ez_y, m_lambda_ez_x, m_lambda_ex_z,  \
        m_lambda_ex_y, m_lambda_ey_x, m_lambda_hz_y, m_lambda_hy_z, m_lambda_hx_z,         \
        m_lambda_hz_x, m_lambda_hy_x, m_lambda_hx_y, eta_ex, eta_ey, eta_ez, eta_hx,       \
        eta_hy, eta_hz, m_eta_ey_z, m_eta_ez_y, m_eta_ez_x, m_eta_ex_z, m_eta_ex_y,        \
        m_eta_ey_x, m_eta_hz_y, m_eta_hy_z, m_eta_hx_z, m_eta_hz_x, m_eta_hy_x,            \
        m_eta_hx_y, adjoint_memory_scratch, ex_s1, ex_s3, ex_fn, ey_s1, ey_s3, ey_fn,      \
        ez_s1, ez_s3, ez_fn, cx_s1, cx_s3, cx_fn, cy_s1, cy_s3, cy_fn, cz_s1, cz_s3,       \
        cz_fn, dex_store, dey_store, dez_store, dcurl_x_store, dcurl_y_store,              \
        dcurl_z_store, grad_f0, grad_df, grad_ca, grad_cb, grad_dca, grad_dcb,             \
        grad_ca_shot, grad_cb_shot, grad_dca_shot, grad_dcb_shot, eta_source_ex,           \
        eta_source_ey, eta_source_ez, az, bz, azh, bzh, ay, by, ayh, byh, ax, bx, axh,     \
        bxh, kz, kzh, ky, kyh, kx, kxh, sources_i, receivers_i, rdz, rdy, rdx, dt, nt,     \
        n_shots, nz, ny, nx, n_sources_per_shot, n_receivers_per_shot, step_ratio,         \
        storage_mode, storage_format, shot_bytes_uncomp, ca_requires_grad,                 \
        cb_requires_grad, dca_requires_grad, dcb_requires_grad, ca_batched, cb_batched,    \
        cq_batched, start_t, pml_z0, pml_y0, pml_x0, pml_z1, pml_y1, pml_x1,               \
        source_component, receiver_component, n_threads, device, execution_backend,        \
        compute_stream, storage_stream);                                                   \
  }

TB3_BORN_DEFINE(2, float)
TB3_BORN_STORE_DEFINE(2, float)
TB3_BGGRAD_DEFINE(2, float)
TB3_BORN_DEFINE(2, double)
TB3_BORN_STORE_DEFINE(2, double)
TB3_BGGRAD_DEFINE(2, double)
TB3_BORN_DEFINE(4, float)
TB3_BORN_STORE_DEFINE(4, float)
TB3_BGGRAD_DEFINE(4, float)
TB3_BORN_DEFINE(4, double)
TB3_BORN_STORE_DEFINE(4, double)
TB3_BGGRAD_DEFINE(4, double)
TB3_BORN_DEFINE(6, float)
TB3_BORN_STORE_DEFINE(6, float)
TB3_BGGRAD_DEFINE(6, float)
TB3_BORN_DEFINE(6, double)
TB3_BORN_STORE_DEFINE(6, double)
TB3_BGGRAD_DEFINE(6, double)
TB3_BORN_DEFINE(8, float)
TB3_BORN_STORE_DEFINE(8, float)
TB3_BGGRAD_DEFINE(8, float)
TB3_BORN_DEFINE(8, double)
TB3_BORN_STORE_DEFINE(8, double)
TB3_BGGRAD_DEFINE(8, double)
