// Stencil-order-2 TM2D kernels (the configuration the benchmarks run).
//
// One code path serves every tile, CPML strips included.  A warp owns 32
// consecutive columns of R consecutive rows: the y-strip state of a row is
// the same for all 32 lanes (uniform branch) and the x-strip state is a
// per-lane branch only in the two column bands of the x strips.  Each kernel
// issues every load it needs -- neighbours, CPML memories and profile values
// included, predicated on the strip state -- before any arithmetic, so a warp
// waits for memory once per launch instead of once per strip row; neighbour
// values are plain cached loads (cheaper here than warp shuffles).
//
// For order 2 the update domain is y in [1, ny), x in [1, nx); H-x only for
// y < ny-1 and H-z only for x < nx-1 (maxwell_tm_core.cuh:454-501).  Every
// expression keeps the generic kernels' operation order, so results are
// bit-identical to them and to the CPU oracle.
#pragma once

#include "tm2d_kernels.cuh"

namespace tb {

// Block coordinates of a tile.  The per-call kernels read them from the
// hardware block index (HwTile: special registers, re-read where used, so they
// hold no registers across the body); the multi-job kernels of the serving
// engine pass a virtual tile (Tile).
struct Tile {
  int x_, y_, z_, gx_, gy_;
  __device__ __forceinline__ int x() const { return x_; }
  __device__ __forceinline__ int y() const { return y_; }
  __device__ __forceinline__ int z() const { return z_; }
  __device__ __forceinline__ int gx() const { return gx_; }
  __device__ __forceinline__ int gy() const { return gy_; }
};
struct HwTile {
  __device__ __forceinline__ int x() const { return (int)blockIdx.x; }
  __device__ __forceinline__ int y() const { return (int)blockIdx.y; }
  __device__ __forceinline__ int z() const { return (int)blockIdx.z; }
  __device__ __forceinline__ int gx() const { return (int)gridDim.x; }
  __device__ __forceinline__ int gy() const { return (int)gridDim.y; }
};

// ---------------------------------------------------------------- forward H
template <typename T, int R, typename TL>
__device__ __forceinline__ void fwd_h_tile(
    const TL tl, const TMGeom<T> &g,
    const T *__restrict__ cq, const T *__restrict__ ey, T *__restrict__ hx,
    T *__restrict__ hz, T *__restrict__ m_ey_x, T *__restrict__ m_ey_z) {
  const int nx = g.nx, ny = g.ny;
  const int x = tl.x() * kTileX + threadIdx.x + 1;
  const int y0 = (tl.y() * kBlockY + threadIdx.y) * R + 1;
  if (y0 >= ny || x >= nx) return;
  const int64_t base = (int64_t)tl.z() * g.N;
  ey += base; hx += base; hz += base; m_ey_x += base; m_ey_z += base;
  if (g.cq_b) cq += base;
  const int j0 = y0 * nx + x;
  {
    // Interior tile (block-uniform): no strip cell for H-x or H-z.
    const int tx0 = tl.x() * kTileX + 1, ty0 = tl.y() * kBlockY * R + 1;
    if (tx0 >= g.pml_x0 && tx0 + kTileX <= g.pml_x1h && ty0 >= g.pml_y0 &&
        ty0 + kBlockY * R <= g.pml_y1h) {
      T e[R + 1], er[R], c[R], vx[R], vz[R];
#pragma unroll
      for (int r = 0; r <= R; ++r) e[r] = ldg(ey + j0 + r * nx);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r * nx;
        er[r] = ldg(ey + j + 1);
        c[r] = ldg(cq + j);
        vx[r] = hx[j];
        vz[r] = hz[j];
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r * nx;
        hx[j] = vx[r] - c[r] * ((e[r + 1] - e[r]) * g.rdy);
        hz[j] = vz[r] + c[r] * ((er[r] - e[r]) * g.rdx);
      }
      return;
    }
  }
  const bool hz_ok = x < nx - 1;
  const bool xs = hz_ok && (x < g.pml_x0 || x >= g.pml_x1h);
  // ---- loads (all issued before any arithmetic)
  T e[R + 1], er[R], c[R], vx[R], vz[R], mz[R], mx[R], pb[R], pa[R], pk[R];
  T qb = 0, qa = 0, qk = 1;
  if (xs) {
    qb = ldg(g.bxh + x);
    qa = ldg(g.axh + x);
    qk = ldg(g.kxh + x);
  }
#pragma unroll
  for (int r = 0; r <= R; ++r) e[r] = (y0 + r < ny) ? ldg(ey + j0 + r * nx) : (T)0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    const bool rv = y < ny, hx_ok = y < ny - 1;
    const bool ys = hx_ok && (y < g.pml_y0 || y >= g.pml_y1h);
    c[r] = rv ? ldg(cq + j) : (T)0;
    vx[r] = hx_ok ? hx[j] : (T)0;
    vz[r] = (rv && hz_ok) ? hz[j] : (T)0;
    er[r] = (rv && hz_ok) ? ldg(ey + j + 1) : (T)0;
    mz[r] = ys ? m_ey_z[j] : (T)0;
    pb[r] = ys ? ldg(g.byh + y) : (T)0;
    pa[r] = ys ? ldg(g.ayh + y) : (T)0;
    pk[r] = ys ? ldg(g.kyh + y) : (T)1;
    mx[r] = (rv && xs) ? m_ey_x[j] : (T)0;
  }
  // ---- arithmetic and stores
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    if (y >= ny) break;
    if (y < ny - 1) {
      T d = (e[r + 1] - e[r]) * g.rdy;
      if (y < g.pml_y0 || y >= g.pml_y1h) {
        const T m = pb[r] * mz[r] + pa[r] * d;
        m_ey_z[j] = m;
        d = d / pk[r] + m;
      }
      hx[j] = vx[r] - c[r] * d;
    }
    if (hz_ok) {
      T d = (er[r] - e[r]) * g.rdx;
      if (xs) {
        const T m = qb * mx[r] + qa * d;
        m_ey_x[j] = m;
        d = d / qk + m;
      }
      hz[j] = vz[r] + c[r] * d;
    }
  }
}
template <typename T, int R>
__global__ void __launch_bounds__(256)
k2_fwd_h(TMGeom<T> g, const T *__restrict__ cq, const T *__restrict__ ey, T *__restrict__ hx,
         T *__restrict__ hz, T *__restrict__ m_ey_x, T *__restrict__ m_ey_z) {
  fwd_h_tile<T, R>(HwTile(), g, cq, ey, hx, hz, m_ey_x, m_ey_z);
}

// ---------------------------------------------------------------- forward E
// Full-grid tiles (32 x 8R) so point entries outside the domain are served.
template <typename T, typename S, int R, int BY = kBlockY, typename TL>
__device__ __forceinline__ void fwd_e_tile(
    const TL tl, const TMGeom<T> &g,
    const T *__restrict__ ca, const T *__restrict__ cb, const T *__restrict__ hx,
    const T *__restrict__ hz, T *__restrict__ ey, T *__restrict__ m_hx_z,
    T *__restrict__ m_hz_x, S *__restrict__ ey_store, S *__restrict__ curl_store,
    PointCSR src, PointCSR rec, const T *__restrict__ f_t, T *__restrict__ r_t) {
  const int nx = g.nx, ny = g.ny;
  const int x = tl.x() * kTileX + threadIdx.x;
  const int y0 = (tl.y() * BY + threadIdx.y) * R;
  const int s = tl.z();
  const int tile = (s * tl.gy() + tl.y()) * tl.gx() + tl.x();
  if (y0 >= ny || x >= nx) return;
  const bool pts = !point_tile_empty(src, rec, tile);
  const int64_t base = (int64_t)s * g.N;
  hx += base; hz += base; ey += base; m_hx_z += base; m_hz_x += base;
  if (g.ca_b) ca += base;
  if (g.cb_b) cb += base;
  if (ey_store) ey_store += base;
  if (curl_store) curl_store += base;
  const int j0 = y0 * nx + x;
  {
    // Interior tile (block-uniform): no strip cell, every cell in the domain.
    const int tx0 = tl.x() * kTileX, ty0 = tl.y() * BY * R;
    if (tx0 >= g.pml_x0 && tx0 + kTileX <= g.pml_x1 && ty0 >= g.pml_y0 &&
        ty0 + BY * R <= g.pml_y1) {
      T vx[R + 1], vz[R], vzl[R], eo[R], a[R], b[R];
#pragma unroll
      for (int r = 0; r <= R; ++r) vx[r] = ldg(hx + j0 + (r - 1) * nx);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r * nx;
        eo[r] = ey[j];
        vz[r] = ldg(hz + j);
        vzl[r] = ldg(hz + j - 1);
        a[r] = ldg(ca + j);
        b[r] = ldg(cb + j);
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r * nx;
        const T curl = (vz[r] - vzl[r]) * g.rdx - (vx[r + 1] - vx[r]) * g.rdy;
        if (ey_store) store_stream(ey_store + j, Codec<S, T>::enc(eo[r]));
        if (curl_store) store_stream(curl_store + j, Codec<S, T>::enc(curl));
        T e = a[r] * eo[r] + b[r] * curl;
        if (pts) e = point_accumulate(src, tile, j, f_t, e);
        ey[j] = e;
        if (pts) point_record(rec, tile, j, r_t, e);
      }
      return;
    }
  }
  const bool xdom = x >= 1;
  const bool xs = xdom && (x < g.pml_x0 || x >= g.pml_x1);
  // ---- loads
  T vx[R + 1], vz[R], vzl[R], eo[R], a[R], b[R], mz[R], mx[R], pb[R], pa[R], pk[R];
  T qb = 0, qa = 0, qk = 1;
  if (xs) {
    qb = ldg(g.bx + x);
    qa = ldg(g.ax + x);
    qk = ldg(g.kx + x);
  }
#pragma unroll
  for (int r = 0; r <= R; ++r) {
    const int y = y0 + r - 1;
    vx[r] = (xdom && y >= 0 && y < ny) ? ldg(hx + j0 + (r - 1) * nx) : (T)0;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    const bool rv = y < ny, dom = rv && xdom && y >= 1;
    const bool ys = dom && (y < g.pml_y0 || y >= g.pml_y1);
    eo[r] = rv ? ey[j] : (T)0;
    vz[r] = dom ? ldg(hz + j) : (T)0;
    vzl[r] = dom ? ldg(hz + j - 1) : (T)0;
    a[r] = dom ? ldg(ca + j) : (T)0;
    b[r] = dom ? ldg(cb + j) : (T)0;
    mz[r] = ys ? m_hx_z[j] : (T)0;
    pb[r] = ys ? ldg(g.by + y) : (T)0;
    pa[r] = ys ? ldg(g.ay + y) : (T)0;
    pk[r] = ys ? ldg(g.ky + y) : (T)1;
    mx[r] = (dom && xs) ? m_hz_x[j] : (T)0;
  }
  // ---- arithmetic and stores
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    if (y >= ny) break;
    const bool dom = xdom && y >= 1;
    T e = eo[r];
    if (dom) {
      T dz = (vz[r] - vzl[r]) * g.rdx;
      T dy = (vx[r + 1] - vx[r]) * g.rdy;
      if (xs) {
        const T m = qb * mx[r] + qa * dz;
        m_hz_x[j] = m;
        dz = dz / qk + m;
      }
      if (y < g.pml_y0 || y >= g.pml_y1) {
        const T m = pb[r] * mz[r] + pa[r] * dy;
        m_hx_z[j] = m;
        dy = dy / pk[r] + m;
      }
      const T curl = dz - dy;
      if (ey_store) store_stream(ey_store + j, Codec<S, T>::enc(e));
      if (curl_store) store_stream(curl_store + j, Codec<S, T>::enc(curl));
      e = a[r] * e + b[r] * curl;
    }
    if (pts) e = point_accumulate(src, tile, j, f_t, e);
    if (dom || pts) ey[j] = e;
    if (pts) point_record(rec, tile, j, r_t, e);
  }
}
template <typename T, typename S, int R, int BY = kBlockY>
__global__ void __launch_bounds__(32 * BY)
k2_fwd_e(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cb, const T *__restrict__ hx,
         const T *__restrict__ hz, T *__restrict__ ey, T *__restrict__ m_hx_z,
         T *__restrict__ m_hz_x, S *__restrict__ ey_store, S *__restrict__ curl_store,
         PointCSR src, PointCSR rec, const T *__restrict__ f_t, T *__restrict__ r_t,
         StepShift sh) {
  if (sh.blk) {
    const int64_t jb = sh.block();
    f_t = shifted(f_t, sh.src, jb);
    r_t = shifted(r_t, sh.rec, jb);
    ey_store = shifted(ey_store, sh.snap, jb);
    curl_store = shifted(curl_store, sh.snap, jb);
  }
  fwd_e_tile<T, S, R, BY>(HwTile(), g, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, ey_store, curl_store,
      src, rec, f_t, r_t);
}

// ---------------------------------------------------------------- adjoint E
// raw_x(x') = q (x' in [pml_x0, pml_x1)) or ax (bx m + q) + q / kx;
// raw_y(y') = -q (y' in [pml_y0, pml_y1)) or ay (by m - q) - q / ky; both 0
// outside the domain (maxwell_tm_cuda_inst.cu:954-994).
template <typename T, int R, int BY = kBlockY, typename TL>
__device__ __forceinline__ void adj_e_tile(
    const TL tl, const TMGeom<T> &g,
    const T *__restrict__ cb, const T *__restrict__ lam_ey,
    T *__restrict__ lam_hx, T *__restrict__ lam_hz, const T *__restrict__ m_hx_z,
    const T *__restrict__ m_hz_x, T *__restrict__ m_hx_z_n, T *__restrict__ m_hz_x_n) {
  const int nx = g.nx, ny = g.ny;
  const int x = tl.x() * kTileX + threadIdx.x + 1;
  const int y0 = (tl.y() * BY + threadIdx.y) * R + 1;
  if (y0 >= ny || x >= nx) return;
  const int64_t base = (int64_t)tl.z() * g.N;
  lam_ey += base; lam_hx += base; lam_hz += base;
  m_hx_z += base; m_hz_x += base; m_hx_z_n += base; m_hz_x_n += base;
  if (g.cb_b) cb += base;
  {
    // Interior tile (block-uniform): cells and their +1 neighbours outside
    // the strips, so raw_x = q and raw_y = -q throughout.
    const int tx0 = tl.x() * kTileX + 1, ty0 = tl.y() * BY * R + 1;
    if (tx0 >= g.pml_x0 && tx0 + kTileX < g.pml_x1 && ty0 >= g.pml_y0 &&
        ty0 + BY * R < g.pml_y1) {
      const int j0 = y0 * nx + x;
      T lq[R + 1], cq_[R + 1], lr[R], cr[R], vx[R], vz[R];
#pragma unroll
      for (int r = 0; r <= R; ++r) {
        lq[r] = ldg(lam_ey + j0 + r * nx);
        cq_[r] = ldg(cb + j0 + r * nx);
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r * nx;
        lr[r] = ldg(lam_ey + j + 1);
        cr[r] = ldg(cb + j + 1);
        vx[r] = lam_hx[j];
        vz[r] = lam_hz[j];
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r * nx;
        const T q = cq_[r] * lq[r], q1 = cq_[r + 1] * lq[r + 1], qr = cr[r] * lr[r];
        lam_hz[j] = vz[r] + ((T)1 * (q - qr)) * g.rdx;
        lam_hx[j] = vx[r] + ((T)1 * ((-q) - (-q1))) * g.rdy;
      }
      return;
    }
  }
  const bool xs = x < g.pml_x0 || x >= g.pml_x1;
  const int xr = x + 1;
  const bool xr_dom = xr < nx;
  const bool xsr = xr_dom && (xr < g.pml_x0 || xr >= g.pml_x1);
  const int j0 = y0 * nx + x;
  // ---- loads
  T lq[R + 1], cbq[R + 1], mz[R + 1], pb[R + 1], pa[R + 1], pk[R + 1];
  T lr[R], cbr[R], mx[R], mxr[R], vx[R], vz[R];
  T qb = 0, qa = 0, qk = 1, rb = 0, ra = 0, rk = 1;
  if (xs) {
    qb = ldg(g.bx + x);
    qa = ldg(g.ax + x);
    qk = ldg(g.kx + x);
  }
  if (xsr) {
    rb = ldg(g.bx + xr);
    ra = ldg(g.ax + xr);
    rk = ldg(g.kx + xr);
  }
#pragma unroll
  for (int r = 0; r <= R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    const bool rv = y < ny;
    const bool ys = rv && (y < g.pml_y0 || y >= g.pml_y1);
    lq[r] = rv ? ldg(lam_ey + j) : (T)0;
    cbq[r] = rv ? ldg(cb + j) : (T)0;
    mz[r] = ys ? ldg(m_hx_z + j) : (T)0;
    pb[r] = ys ? ldg(g.by + y) : (T)0;
    pa[r] = ys ? ldg(g.ay + y) : (T)0;
    pk[r] = ys ? ldg(g.ky + y) : (T)1;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    const bool rv = y < ny;
    vx[r] = rv ? lam_hx[j] : (T)0;
    vz[r] = rv ? lam_hz[j] : (T)0;
    mx[r] = (rv && xs) ? ldg(m_hz_x + j) : (T)0;
    lr[r] = (rv && xr_dom) ? ldg(lam_ey + j + 1) : (T)0;
    cbr[r] = (rv && xr_dom) ? ldg(cb + j + 1) : (T)0;
    mxr[r] = (rv && xsr) ? ldg(m_hz_x + j + 1) : (T)0;
  }
  // ---- arithmetic and stores
  T q[R + 1], ry[R + 1];
#pragma unroll
  for (int r = 0; r <= R; ++r) {
    const int y = y0 + r;
    q[r] = cbq[r] * lq[r];
    if (y >= ny) {
      ry[r] = (T)0;
    } else if (y >= g.pml_y0 && y < g.pml_y1) {
      ry[r] = -q[r];
    } else {
      const T mn = pb[r] * mz[r] - q[r];
      ry[r] = pa[r] * mn - q[r] / pk[r];
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    if (y >= ny) break;
    T rx, rxr;
    if (!xs) {
      rx = q[r];
    } else {
      const T mn = qb * mx[r] + q[r];
      rx = qa * mn + q[r] / qk;
      m_hz_x_n[j] = mn;
    }
    if (!xr_dom) {
      rxr = (T)0;
    } else {
      const T qr = cbr[r] * lr[r];
      if (!xsr) {
        rxr = qr;
      } else {
        const T mn = rb * mxr[r] + qr;
        rxr = ra * mn + qr / rk;
      }
    }
    if (y < g.pml_y0 || y >= g.pml_y1) m_hx_z_n[j] = pb[r] * mz[r] - q[r];
    const T ax_ = (T)1 * (rx - rxr);
    lam_hz[j] = vz[r] + ax_ * g.rdx;
    const T ay_ = (T)1 * (ry[r] - ry[r + 1]);
    lam_hx[j] = vx[r] + ay_ * g.rdy;
  }
}
template <typename T, int R, int BY = kBlockY>
__global__ void __launch_bounds__(32 * BY)
k2_adj_e(TMGeom<T> g, const T *__restrict__ cb, const T *__restrict__ lam_ey,
         T *__restrict__ lam_hx, T *__restrict__ lam_hz, const T *__restrict__ m_hx_z,
         const T *__restrict__ m_hz_x, T *__restrict__ m_hx_z_n, T *__restrict__ m_hz_x_n) {
  adj_e_tile<T, R, BY>(HwTile(), g, cb, lam_ey, lam_hx, lam_hz, m_hx_z, m_hz_x, m_hx_z_n,
      m_hz_x_n);
}

// ---------------------------------------------------------------- adjoint H
// raw_eyz(y') = adj (y' in [pml_y0, pml_y1h)) or ayh (byh m + adj) + adj / kyh,
// adj = -cq lam_hx, 0 unless y' in [1, ny-1); raw_eyx(x') likewise with
// adj = cq lam_hz, 0 unless x' in [1, nx-1) (maxwell_tm_cuda_inst.cu:1082-1122).
//
// Adjoint H-phase interior update of U consecutive shots starting at s0 (see
// k2_adj_h): loads of all U shots first, then arithmetic, stores and the
// per-row image sums sa/sb (shot order preserved).
template <typename T, typename S, int R, int U>
__device__ __forceinline__ void adj_h_interior_group(
    const TMGeom<T> &g, const GradArgs<T, S> &ga, const T *__restrict__ lam_hx,
    const T *__restrict__ lam_hz, T *__restrict__ lam_ey, const PointCSR &rec,
    const PointCSR &src, const unsigned char *__restrict__ rowf, const T *__restrict__ gr_t,
    T *__restrict__ gf_t, int s0, int tiles_per_shot, int tile_xy, int j0, int trow_stride,
    const T (&a)[R], const T (&cz)[R + 1],
    const T (&cx)[R], const T (&cl)[R], T (&sa)[R], T (&sb)[R]) {
  const int nx = g.nx;
  T hxz[U][R + 1], hzx[U][R], hzl[U][R], lam[U][R];
  S ev[U][R], cv[U][R];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int64_t base = (int64_t)(s0 + u) * g.N;
    const int64_t sbase = ga.snap_base(s0 + u, g.N);
#pragma unroll
    for (int r = 0; r <= R; ++r) hxz[u][r] = ldg(lam_hx + base + j0 + (r - 1) * nx);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t i = base + j0 + r * nx;
      lam[u][r] = lam_ey[i];
      hzx[u][r] = ldg(lam_hz + i);
      hzl[u][r] = ldg(lam_hz + i - 1);
      ev[u][r] = ga.ey_st ? load_stream(ga.ey_st + sbase + j0 + r * nx) : S(0.f);
      cv[u][r] = ga.cu_st ? load_stream(ga.cu_st + sbase + j0 + r * nx) : S(0.f);
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int s = s0 + u;
    const int64_t base = (int64_t)s * g.N;
    const int tile = s * tiles_per_shot + tile_xy;
    const bool pts = rowf != nullptr && __ldg(rowf + s * trow_stride) != 0 &&
                     !point_tile_empty(src, rec, tile);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r * nx;
      const T rz0 = -cz[r] * hxz[u][r], rz1 = -cz[r + 1] * hxz[u][r + 1];
      const T rx = cx[r] * hzx[u][r], rxl = cl[r] * hzl[u][r];
      T v = a[r] * lam[u][r];
      v = v + (((T)1 * (rz0 - rz1)) * g.rdy + ((T)1 * (rxl - rx)) * g.rdx);
      if (pts) v = point_accumulate(rec, tile, j, gr_t, v);
      lam_ey[base + j] = v;
      if (pts) point_record(src, tile, j, gf_t, v);
      if (ga.ey_st) {
        const T t = v * Codec<S, T>::dec(ev[u][r]) * ga.kscale;
        if (ga.batched_ca) ga.grad_ca[base + j] = ga.grad_ca[base + j] + t;
        else sa[r] = sa[r] + t;
      }
      if (ga.cu_st) {
        const T t = v * Codec<S, T>::dec(cv[u][r]) * ga.kscale;
        if (ga.batched_cb) ga.grad_cb[base + j] = ga.grad_cb[base + j] + t;
        else sb[r] = sb[r] + t;
      }
    }
  }
}

// Full-grid tiles (32 x BY R, BY warps per block).  Each thread loops over the
// shots of the call: model coefficients are read once, and the image terms
// lam * Ey^t * k and lam * curlH^t * k of all shots are summed before one
// read-modify-write of the model gradient (batched models keep one gradient
// per shot).
template <typename T, typename S, int R, int BY = kBlockY, typename TL>
__device__ __forceinline__ void adj_h_tile(
    const TL tl, const TMGeom<T> &g,
    const T *__restrict__ ca, const T *__restrict__ cq,
    const T *__restrict__ lam_hx, const T *__restrict__ lam_hz, T *__restrict__ lam_ey,
    const T *__restrict__ m_ey_x, const T *__restrict__ m_ey_z, T *__restrict__ m_ey_x_n,
    T *__restrict__ m_ey_z_n, PointCSR rec, PointCSR src,
    const unsigned char *__restrict__ rowf, const T *__restrict__ gr_t,
    T *__restrict__ gf_t, GradArgs<T, S> ga) {
  const int nx = g.nx, ny = g.ny;
  const int x = tl.x() * kTileX + threadIdx.x;
  const int y0 = (tl.y() * BY + threadIdx.y) * R;
  if (y0 >= ny || x >= nx) return;
  const int tile_xy = tl.y() * tl.gx() + tl.x();
  const int tiles_per_shot = tl.gx() * tl.gy();
  const bool xdom = x >= 1;
  const bool rx_ok = x >= 1 && x < nx - 1;  // raw_eyx defined at x
  const bool xs = rx_ok && (x < g.pml_x0 || x >= g.pml_x1h);
  const int xl = x - 1;
  const bool rxl_ok = xl >= 1 && xl < nx - 1;  // ... and at x - 1
  const bool xsl = rxl_ok && (xl < g.pml_x0 || xl >= g.pml_x1h);
  const int j0 = y0 * nx + x;
  const bool imaging = ga.ey_st != nullptr || ga.cu_st != nullptr;
  {
    // Interior tile (block-uniform): cells and their -1 neighbours outside
    // the strips, unbatched coefficients.
    const int tx0 = tl.x() * kTileX, ty0 = tl.y() * BY * R;
    if (!g.ca_b && !g.cq_b && tx0 - 1 >= g.pml_x0 && tx0 + kTileX <= g.pml_x1h &&
        ty0 - 1 >= g.pml_y0 && ty0 + BY * R <= g.pml_y1h) {
      T a[R], cz[R + 1], cx[R], cl[R], sa[R], sb[R];
#pragma unroll
      for (int r = 0; r <= R; ++r) cz[r] = ldg(cq + j0 + (r - 1) * nx);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r * nx;
        a[r] = ldg(ca + j);
        cx[r] = ldg(cq + j);
        cl[r] = ldg(cq + j - 1);
        sa[r] = sb[r] = (T)0;
      }
      // Shots in groups of U: all loads of a group are issued before its
      // arithmetic so U shots' memory latency overlaps.
      constexpr int U = 4;
      const unsigned char *rowf_t = rowf ? rowf + tl.y() : nullptr;
      int s0 = 0;
      for (; s0 + U <= g.n_shots; s0 += U)
        adj_h_interior_group<T, S, R, U>(g, ga, lam_hx, lam_hz, lam_ey, rec, src, rowf_t, gr_t,
                                         gf_t, s0, tiles_per_shot, tile_xy, j0, tl.gy(), a, cz, cx,
                                         cl, sa, sb);
      for (; s0 < g.n_shots; ++s0)
        adj_h_interior_group<T, S, R, 1>(g, ga, lam_hx, lam_hz, lam_ey, rec, src, rowf_t, gr_t,
                                         gf_t, s0, tiles_per_shot, tile_xy, j0, tl.gy(), a, cz, cx,
                                         cl, sa, sb);
      if (imaging) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r * nx;
          if (ga.ey_st && !ga.batched_ca) ga.grad_ca[j] = ga.grad_ca[j] + sa[r];
          if (ga.cu_st && !ga.batched_cb) ga.grad_cb[j] = ga.grad_cb[j] + sb[r];
        }
      }
      return;
    }
  }
  // Shot-independent loads: coefficients (unless batched) and profiles.
  T qb = 0, qa = 0, qk = 1, lb = 0, la = 0, lk = 1;
  if (xs) {
    qb = ldg(g.bxh + x);
    qa = ldg(g.axh + x);
    qk = ldg(g.kxh + x);
  }
  if (xsl) {
    lb = ldg(g.bxh + xl);
    la = ldg(g.axh + xl);
    lk = ldg(g.kxh + xl);
  }
  T a[R], cqz[R + 1], cqx[R], cql[R], pb[R + 1], pa[R + 1], pk[R + 1];
  bool zok[R + 1], zs[R + 1];
#pragma unroll
  for (int r = 0; r <= R; ++r) {  // rows y0-1 .. y0+R-1 for raw_eyz
    const int y = y0 + r - 1;
    zok[r] = xdom && y >= 1 && y < ny - 1;
    zs[r] = zok[r] && (y < g.pml_y0 || y >= g.pml_y1h);
    cqz[r] = (zok[r] && !g.cq_b) ? ldg(cq + j0 + (r - 1) * nx) : (T)0;
    pb[r] = zs[r] ? ldg(g.byh + y) : (T)0;
    pa[r] = zs[r] ? ldg(g.ayh + y) : (T)0;
    pk[r] = zs[r] ? ldg(g.kyh + y) : (T)1;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r, j = j0 + r * nx;
    const bool rv = y < ny;
    const bool ok = rv && y >= 1;
    a[r] = (ok && xdom && !g.ca_b) ? ldg(ca + j) : (T)0;
    cqx[r] = (ok && rx_ok && !g.cq_b) ? ldg(cq + j) : (T)0;
    cql[r] = (ok && rxl_ok && !g.cq_b) ? ldg(cq + j - 1) : (T)0;
  }
  T sum_ca[R], sum_cb[R];
#pragma unroll
  for (int r = 0; r < R; ++r) sum_ca[r] = sum_cb[r] = (T)0;
#pragma unroll 1
  for (int s = 0; s < g.n_shots; ++s) {
    const int64_t base = (int64_t)s * g.N;
    const int tile = s * tiles_per_shot + tile_xy;
    const bool pts = rowf != nullptr && __ldg(rowf + s * tl.gy() + tl.y()) != 0 &&
                     !point_tile_empty(src, rec, tile);
    const T *lhx = lam_hx + base, *lhz = lam_hz + base, *mex = m_ey_x + base;
    const T *mez = m_ey_z + base;
    T *ley = lam_ey + base;
    const int64_t sbase = ga.snap_base(s, g.N);
    const S *est = ga.ey_st ? ga.ey_st + sbase : nullptr;
    const S *cst = ga.cu_st ? ga.cu_st + sbase : nullptr;
    // ---- loads for this shot
    T hxz[R + 1], mz[R + 1], cz[R + 1], hzx[R], hzl[R], mx[R], ml[R], lam[R], as[R];
    T cx[R], cl[R];
    S ev[R], cv[R];
#pragma unroll
    for (int r = 0; r <= R; ++r) {
      const int j = j0 + (r - 1) * nx;
      hxz[r] = zok[r] ? ldg(lhx + j) : (T)0;
      mz[r] = zs[r] ? ldg(mez + j) : (T)0;
      cz[r] = (zok[r] && g.cq_b) ? ldg(cq + base + j) : cqz[r];
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int y = y0 + r, j = j0 + r * nx;
      const bool rv = y < ny;
      const bool ok = rv && y >= 1;
      lam[r] = rv ? ley[j] : (T)0;
      hzx[r] = (ok && rx_ok) ? ldg(lhz + j) : (T)0;
      hzl[r] = (ok && rxl_ok) ? ldg(lhz + j - 1) : (T)0;
      mx[r] = (ok && xs) ? ldg(mex + j) : (T)0;
      ml[r] = (ok && xsl) ? ldg(mex + j - 1) : (T)0;
      as[r] = (ok && xdom && g.ca_b) ? ldg(ca + base + j) : a[r];
      cx[r] = (ok && rx_ok && g.cq_b) ? ldg(cq + base + j) : cqx[r];
      cl[r] = (ok && rxl_ok && g.cq_b) ? ldg(cq + base + j - 1) : cql[r];
      const bool im = imaging && ok && xdom;
      ev[r] = (im && est) ? load_stream(est + j) : S(0.f);
      cv[r] = (im && cst) ? load_stream(cst + j) : S(0.f);
    }
    // ---- arithmetic and stores
    T rz[R + 1];
#pragma unroll
    for (int r = 0; r <= R; ++r) {
      const int y = y0 + r - 1;
      const T adj = -cz[r] * hxz[r];
      if (!zok[r]) {
        rz[r] = (T)0;
      } else if (!zs[r]) {
        rz[r] = adj;
      } else {
        const T mn = pb[r] * mz[r] + adj;
        rz[r] = pa[r] * mn + adj / pk[r];
        if (r >= 1) m_ey_z_n[base + j0 + (r - 1) * nx] = mn;  // own row y
      }
      (void)y;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int y = y0 + r, j = j0 + r * nx;
      if (y >= ny) break;
      const bool dom = xdom && y >= 1;
      if (!dom && !pts) continue;
      T v = lam[r];
      if (dom) {
        T rx = (T)0, rxl = (T)0;
        if (rx_ok) {
          const T adj = cx[r] * hzx[r];
          if (!xs) {
            rx = adj;
          } else {
            const T mn = qb * mx[r] + adj;
            rx = qa * mn + adj / qk;
            m_ey_x_n[base + j] = mn;
          }
        }
        if (rxl_ok) {
          const T adj = cl[r] * hzl[r];
          if (!xsl) {
            rxl = adj;
          } else {
            const T mn = lb * ml[r] + adj;
            rxl = la * mn + adj / lk;
          }
        }
        v = as[r] * v;
        const T dz = (T)1 * (rz[r] - rz[r + 1]);
        const T dx = (T)1 * (rxl - rx);
        v = v + (dz * g.rdy + dx * g.rdx);
      }
      if (pts) v = point_accumulate(rec, tile, j, gr_t, v);
      ley[j] = v;
      if (pts) point_record(src, tile, j, gf_t, v);
      if (imaging && dom) {
        if (est) {
          const T t = v * Codec<S, T>::dec(ev[r]) * ga.kscale;
          if (ga.batched_ca) ga.grad_ca[base + j] = ga.grad_ca[base + j] + t;
          else sum_ca[r] = sum_ca[r] + t;
        }
        if (cst) {
          const T t = v * Codec<S, T>::dec(cv[r]) * ga.kscale;
          if (ga.batched_cb) ga.grad_cb[base + j] = ga.grad_cb[base + j] + t;
          else sum_cb[r] = sum_cb[r] + t;
        }
      }
    }
  }
  if (!imaging || !xdom) return;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    if (y >= ny) break;
    if (y < 1) continue;
    const int j = j0 + r * nx;
    if (ga.ey_st && !ga.batched_ca) ga.grad_ca[j] = ga.grad_ca[j] + sum_ca[r];
    if (ga.cu_st && !ga.batched_cb) ga.grad_cb[j] = ga.grad_cb[j] + sum_cb[r];
  }
}
// 64 registers per thread at any block height (4 blocks of 8 warps or 8 of 4
// per SM); the compiler's own choice spills.
template <typename T, typename S, int R, int BY>
__global__ void __launch_bounds__(32 * BY, 32 / BY)
k2_adj_h(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cq,
         const T *__restrict__ lam_hx, const T *__restrict__ lam_hz, T *__restrict__ lam_ey,
         const T *__restrict__ m_ey_x, const T *__restrict__ m_ey_z, T *__restrict__ m_ey_x_n,
         T *__restrict__ m_ey_z_n, PointCSR rec, PointCSR src,
         const unsigned char *__restrict__ rowf, const T *__restrict__ gr_t,
         T *__restrict__ gf_t, GradArgs<T, S> ga, StepShift sh) {
  if (sh.blk) {
    const int64_t jb = sh.block();
    gr_t = shifted(gr_t, sh.rec, jb);
    gf_t = shifted(gf_t, sh.src, jb);
    ga.ey_st = shifted(ga.ey_st, sh.snap, jb);
    ga.cu_st = shifted(ga.cu_st, sh.snap, jb);
  }
  adj_h_tile<T, S, R, BY>(HwTile(), g, ca, cq, lam_hx, lam_hz, lam_ey, m_ey_x, m_ey_z, m_ey_x_n,
      m_ey_z_n, rec, src, rowf, gr_t, gf_t, ga);
}

}  // namespace tb
