// Fused one-launch-per-step TM2D forward for stencil order 2 in FP32.
//
// Layout.  The kernels work on a pitched internal copy of the state: every
// field of a shot is ny rows of `pitch` floats, column x at pitched column
// x + padl, shots one after the other, and one guard row before and after
// each array so that the neighbours of the first and last rows (read, never
// used) stay in bounds.  padl puts the first interior column on a 128-byte
// boundary; the model coefficients get the same layout.  A thread owns four
// consecutive columns (one float4) and walks down kF4Rows rows.
//
// Fusion.  Both half steps of a time step run in one pass: walking down, a
// thread keeps Ey(y) and the new H-x of row y-1 in registers, computes the
// new H-x and H-z of row y, recomputes the new H-z of column x-1 (owned by
// the neighbouring thread) from the old state, and then updates Ey(y).
// Reading old and writing new values in the same arrays would race between
// threads, so Ey, H-x, H-z and the two H-phase CPML memories ping-pong
// between two complete copies; the two E-phase CPML memories are read and
// written by their own cell's thread only and are updated in place.  Every
// row is stored whole (cells a step does not update keep their old value),
// so both copies stay consistent.  Each field crosses HBM once per step.
//
// Work split.  Columns [xl, xr) (no CPML x-strip, no x edge among the cells a
// thread updates or recomputes) run with warps of 128 columns: interior rows
// [yt, yb) in straight-line code, the top and bottom bands (the y strips and
// the y edges) in the same code with row-uniform CPML branches.  The side
// columns (x strips, x edges, padding) run in blocks whose warps are four
// independent strands of 8 lanes (32 columns), with per-cell masks.  All three
// kinds of block belong to one launch, touch disjoint cells and read only the
// old copy.
//
// Snapshots (caller layout, rows of nx cells at any alignment) are written
// through a per-warp shared-memory transpose, so every store instruction
// writes consecutive cells.
//
// The loads of row y+1 are issued before row y is computed (one row of
// prefetch), with 128-bit loads and stores throughout; neighbours at x-1 and
// x+4 are 32-bit loads that hit L1.  Every value is computed with the same
// operations in the same order as the two-kernel path (tm2d_s2.cuh), so
// results are bit-identical to it and to the CPU oracle.
#pragma once

#include "tm2d_kernels.cuh"

namespace tb {

constexpr int kF4Warps = 4;  // warps per block
constexpr int kF4Rows = 2;   // rows per interior thread (segment height)
constexpr int kF4FRows = 1;  // rows per frame strand: one load round trip per task
constexpr int kF4PtW = 32;   // point tiles: 32 pitched columns ...
constexpr int kF4PtH = 8;    // ... by 8 rows

// Decomposition of one shot's grid for the fused kernels (host-computed).
struct F4Geom {
  int pitch, padl;         // row pitch (floats); column x sits at pitched column x + padl
  int64_t pshot;           // floats per shot
  int xl, xr;              // column band [xl, xr): (xl + padl) % 32 == 0, (xr - xl) % 4 == 0
  int yt, yb;              // interior rows [yt, yb): (yb - yt) % kF4Rows == 0
  int n_ix;                // warps across the column band (128 columns each)
  int n_iseg;              // interior row segments
  int n_btop, n_bbot;      // band row segments: top [0, yt), bottom [yb, ny)
  int n_chunks;            // 32-column chunks of a pitched row
  int n_lchunk, r_chunk0;  // side chunks: [0, n_lchunk) and [r_chunk0, n_chunks)
  int n_schunk, n_sseg;    // side chunks; side row segments (kF4FRows rows)
  PointTiles pt;           // point-list tiles
};

// In/out state of one fused forward step (pitched arrays, shot 0 row 0).
// mex = m_ey_x, mez = m_ey_z (H phase); mhx = m_hx_z, mhz = m_hz_x (E phase).
template <typename T> struct FwdState {
  const T *ey, *hx, *hz, *mex, *mez, *mhx, *mhz;          // old (read)
  T *ey_n, *hx_n, *hz_n, *mex_n, *mez_n, *mhx_n, *mhz_n;  // new (written)
};

struct V4 {
  float c[4];
};
__device__ __forceinline__ V4 ldv(const float *p) {
  const float4 t = __ldg(reinterpret_cast<const float4 *>(p));
  return V4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ V4 ldv_rw(const float *p) {  // buffer also written by this kernel
  const float4 t = *reinterpret_cast<const float4 *>(p);
  return V4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void stv(float *p, const V4 &v) {
  *reinterpret_cast<float4 *>(p) = make_float4(v.c[0], v.c[1], v.c[2], v.c[3]);
}

// Point entries of `tile` at cells cell0 + lo .. cell0 + hi - 1 of one row:
// v[c] = v[c] + vals[e] in entry order (as point_accumulate per cell).
__device__ __forceinline__ void points_add4(const PointCSR &pl, int tile, int cell0, int lo,
                                            int hi, const float *vals, V4 &v) {
  if (pl.start == nullptr || vals == nullptr) return;
  const int b = __ldg(pl.start + tile), e = __ldg(pl.start + tile + 1);
  for (int k = b; k < e; ++k) {
    const int d = __ldg(pl.cell + k) - cell0;
    if (d >= lo && d < hi) {
      const float f = __ldg(vals + __ldg(pl.ent + k));
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (d == c) v.c[c] = v.c[c] + f;
    }
  }
}
__device__ __forceinline__ void points_rec4(const PointCSR &pl, int tile, int cell0, int lo,
                                            int hi, float *out, const V4 &v) {
  if (pl.start == nullptr || out == nullptr) return;
  const int b = __ldg(pl.start + tile), e = __ldg(pl.start + tile + 1);
  for (int k = b; k < e; ++k) {
    const int d = __ldg(pl.cell + k) - cell0;
    if (d >= lo && d < hi) {
      float w = v.c[0];
#pragma unroll
      for (int c = 1; c < 4; ++c)
        if (d == c) w = v.c[c];
      out[__ldg(pl.ent + k)] = w;
    }
  }
}

__device__ __forceinline__ int f4_tile(const F4Geom &q, int s, int y, int jx) {
  return (s * q.pt.tiles_y + y / kF4PtH) * q.pt.tiles_x + jx / kF4PtW;
}

// Does tile row y / kF4PtH of shot s hold any point (row-uniform test)?
__device__ __forceinline__ bool f4_row_points(const F4Geom &q, const unsigned char *rowf, int s,
                                              int y) {
  return rowf != nullptr && __ldg(rowf + s * q.pt.tiles_y + y / kF4PtH) != 0;
}

__device__ __forceinline__ float sel(bool p, float a, float b) { return p ? a : b; }

// d / k for a CPML kappa k > 0.  A zero numerator (a field the wave has not
// reached) would take the IEEE division's slow path; it divides 1 instead
// and returns d, which equals d / k (signed zero included) for k > 0.
__device__ __forceinline__ float div_k(float d, float k) {
  const float q = (d == 0.f ? 1.f : d) / k;
  return d == 0.f ? d : q;
}

// Per-shot pointers of the step state.
__device__ __forceinline__ FwdState<float> shot_state(const FwdState<float> &st, int64_t b) {
  return FwdState<float>{st.ey + b,    st.hx + b,    st.hz + b,    st.mex + b,   st.mez + b,
                         st.mhx + b,   st.mhz + b,   st.ey_n + b,  st.hx_n + b,  st.hz_n + b,
                         st.mex_n + b, st.mez_n + b, st.mhx_n + b, st.mhz_n + b};
}

// Snapshot row of a warp: lane l holds cells 4l .. 4l+3 of the warp's row
// segment (starting at global cell `dst0`); the first `nvalid` cells are
// written, 32 consecutive cells per store instruction.  Every lane of the
// warp must call it.
template <typename S> struct Pack4;
template <> struct Pack4<float> {
  __device__ static __forceinline__ void put(float *sb, const V4 &v) {
    *reinterpret_cast<float4 *>(sb) = make_float4(v.c[0], v.c[1], v.c[2], v.c[3]);
  }
};
template <> struct Pack4<__nv_bfloat16> {
  __device__ static __forceinline__ void put(__nv_bfloat16 *sb, const V4 &v) {
    const __nv_bfloat162 lo = __halves2bfloat162(__float2bfloat16(v.c[0]), __float2bfloat16(v.c[1]));
    const __nv_bfloat162 hi = __halves2bfloat162(__float2bfloat16(v.c[2]), __float2bfloat16(v.c[3]));
    uint2 u;
    u.x = *reinterpret_cast<const unsigned *>(&lo);
    u.y = *reinterpret_cast<const unsigned *>(&hi);
    *reinterpret_cast<uint2 *>(sb) = u;
  }
};
template <typename S>
__device__ __forceinline__ void snap_row(S *sb, S *dst0, int nvalid, const V4 &v) {
  Pack4<S>::put(sb + 4 * threadIdx.x, v);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int m = 32 * k + threadIdx.x;
    if (m < nvalid) store_stream(dst0 + m, sb[m]);
  }
  __syncwarp();
}

// ---------------------------------------------------------------- column band
// Loads of one row y of the walk (j = pitched index of (y, x)).
struct FwdRow {
  V4 e1, hx, hz, cq, ca, cb;  // Ey(y+1); H-x, H-z, coefficients at y
  float er, el, hzl, cql;     // Ey(y, x+4), Ey(y, x-1), H-z(y, x-1), cq(y, x-1)
  V4 mez, mhx;                // y-strip memories (band rows only)
};
template <bool YS>
__device__ __forceinline__ void load_row(FwdRow &L, const TMGeom<float> &g,
                                         const FwdState<float> &st, const float *ca,
                                         const float *cb, const float *cq, int j, int pitch,
                                         int y) {
  L.e1 = ldv(st.ey + j + pitch);
  L.hx = ldv(st.hx + j);
  L.hz = ldv(st.hz + j);
  L.cq = ldv(cq + j);
  L.ca = ldv(ca + j);
  L.cb = ldv(cb + j);
  L.er = __ldg(st.ey + j + 4);
  L.el = __ldg(st.ey + j - 1);
  L.hzl = __ldg(st.hz + j - 1);
  L.cql = __ldg(cq + j - 1);
  if (YS) {
    const V4 zero{{0.f, 0.f, 0.f, 0.f}};
    const bool zs = y >= 1 && y < g.ny - 1 && (y < g.pml_y0 || y >= g.pml_y1h);
    const bool ys = y >= 1 && (y < g.pml_y0 || y >= g.pml_y1);
    L.mez = zs ? ldv(st.mez + j) : zero;
    L.mhx = ys ? ldv_rw(st.mhx + j) : zero;
  }
}

// Columns [xl, xr).  YS = false: interior row segments (no strip, no edge;
// straight-line code).  YS = true: band row segments (y strips and y edges,
// row-uniform branches).  Grid: (n_ix, ceil(segments / kF4Warps), shots);
// block (32, kF4Warps).  Lanes past xr repeat the last live lane's columns
// without storing, so that every lane takes part in the snapshot transpose.
template <typename S, bool YS>
__device__ __forceinline__ void f4_fwd_cols_body(
    const TMGeom<float> &g, const F4Geom &q, const float *__restrict__ ca,
    const float *__restrict__ cb, const float *__restrict__ cq, const FwdState<float> &st0,
    S *__restrict__ est, S *__restrict__ cst, const PointCSR &src, const PointCSR &rec,
    const unsigned char *rowf, const float *__restrict__ f_t, float *__restrict__ r_t, int bx,
    int by, S *sb_e, S *sb_c) {
  constexpr int RS = kF4Rows;
  const int seg = by * kF4Warps + threadIdx.y;
  int y0, yend;
  if (!YS) {
    if (seg >= q.n_iseg) return;
    y0 = q.yt + seg * RS;
    yend = y0 + RS;
  } else {
    if (seg >= q.n_btop + q.n_bbot) return;
    if (seg < q.n_btop) {
      y0 = seg * RS;
      yend = min(y0 + RS, q.yt);
    } else {
      y0 = q.yb + (seg - q.n_btop) * RS;
      yend = min(y0 + RS, g.ny);
    }
  }
  const int xw = q.xl + bx * 128;  // first column of the warp
  const int n_live = min(32, (q.xr - xw) / 4);
  const bool live = (int)threadIdx.x < n_live;
  const int x = xw + 4 * min((int)threadIdx.x, n_live - 1);
  const int s = blockIdx.z;
  const int64_t base = (int64_t)s * q.pshot;
  const FwdState<float> st = shot_state(st0, base);
  if (g.ca_b) ca += base;
  if (g.cb_b) cb += base;
  if (g.cq_b) cq += base;
  const int nx = g.nx, ny = g.ny, pitch = q.pitch;
  const int64_t cbase = (int64_t)s * g.N;  // caller layout (snapshots)
  const int jx = x + q.padl;
  const float rdy = g.rdy, rdx = g.rdx;

  // Prologue: Ey(y0) and the new H-x of row y0-1.
  int j = (y0 - 1) * pitch + jx;
  V4 e0, hxp;
  {
    const V4 em = ldv(st.ey + j), h = ldv(st.hx + j), c = ldv(cq + j);
    e0 = ldv(st.ey + j + pitch);
    const int y = y0 - 1;
    hxp = h;
    if (!YS || (y >= 1 && y < ny - 1)) {
      V4 d;
#pragma unroll
      for (int k = 0; k < 4; ++k) d.c[k] = (e0.c[k] - em.c[k]) * rdy;
      if (YS && (y < g.pml_y0 || y >= g.pml_y1h)) {
        const V4 mz = ldv(st.mez + j);
        const float zb = __ldg(g.byh + y), za = __ldg(g.ayh + y), zk = __ldg(g.kyh + y);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float m = zb * mz.c[k] + za * d.c[k];
          d.c[k] = div_k(d.c[k], zk) + m;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) hxp.c[k] = h.c[k] - c.c[k] * d.c[k];
    }
  }
  j += pitch;
  FwdRow nxt;
  load_row<YS>(nxt, g, st, ca, cb, cq, j, pitch, y0);
#pragma unroll
  for (int r = 0; r < RS; ++r) {
    const int y = y0 + r;
    if (YS && y >= yend) break;
    const FwdRow L = nxt;
    if (r + 1 < RS && (!YS || y + 1 < yend))
      load_row<YS>(nxt, g, st, ca, cb, cq, j + pitch, pitch, y + 1);
    const bool hxu = !YS || (y >= 1 && y < ny - 1);
    const bool zs = YS && hxu && (y < g.pml_y0 || y >= g.pml_y1h);
    const bool yh = !YS || y >= 1;
    const bool ys = YS && yh && (y < g.pml_y0 || y >= g.pml_y1);
    // ---- H-x
    V4 hxn = L.hx;
    if (hxu) {
      V4 d;
#pragma unroll
      for (int k = 0; k < 4; ++k) d.c[k] = (L.e1.c[k] - e0.c[k]) * rdy;
      if (zs) {
        const float zb = __ldg(g.byh + y), za = __ldg(g.ayh + y), zk = __ldg(g.kyh + y);
        V4 mn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          mn.c[k] = zb * L.mez.c[k] + za * d.c[k];
          d.c[k] = div_k(d.c[k], zk) + mn.c[k];
        }
        if (live) stv(st.mez_n + j, mn);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) hxn.c[k] = L.hx.c[k] - L.cq.c[k] * d.c[k];
    }
    // ---- H-z (columns x .. x+3 and x-1) and E
    V4 hzn = L.hz, en = e0;
    if (yh) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float er = k < 3 ? e0.c[k < 3 ? k + 1 : 3] : L.er;
        hzn.c[k] = L.hz.c[k] + L.cq.c[k] * ((er - e0.c[k]) * rdx);
      }
      const float hznl = L.hzl + L.cql * ((e0.c[0] - L.el) * rdx);
      V4 curl;
      if (!ys) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float left = k ? hzn.c[k ? k - 1 : 0] : hznl;
          curl.c[k] = (hzn.c[k] - left) * rdx - (hxn.c[k] - hxp.c[k]) * rdy;
        }
      } else {
        const float yb = __ldg(g.by + y), ya = __ldg(g.ay + y), yk = __ldg(g.ky + y);
        V4 mn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float left = k ? hzn.c[k ? k - 1 : 0] : hznl;
          const float dz = (hzn.c[k] - left) * rdx;
          float dy = (hxn.c[k] - hxp.c[k]) * rdy;
          mn.c[k] = yb * L.mhx.c[k] + ya * dy;
          dy = div_k(dy, yk) + mn.c[k];
          curl.c[k] = dz - dy;
        }
        if (live) stv(st.mhx_n + j, mn);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) en.c[k] = L.ca.c[k] * e0.c[k] + L.cb.c[k] * curl.c[k];
      const int64_t row0 = cbase + (int64_t)y * nx + xw;
      if (est) snap_row(sb_e, est + row0, 4 * n_live, e0);
      if (cst) snap_row(sb_c, cst + row0, 4 * n_live, curl);
    }
    const int tile = f4_tile(q, s, y, jx);
    const bool pts = f4_row_points(q, rowf, s, y) && live && !point_tile_empty(src, rec, tile);
    if (pts) points_add4(src, tile, y * nx + x, 0, 4, f_t, en);
    if (live) {
      stv(st.hx_n + j, hxn);
      stv(st.hz_n + j, hzn);
      stv(st.ey_n + j, en);
    }
    if (pts) points_rec4(rec, tile, y * nx + x, 0, 4, r_t, en);
    hxp = hxn;
    e0 = L.e1;
    j += pitch;
  }
}

// ---------------------------------------------------------------- side columns
// Grid: (ceil(n_sseg / (4 kF4Warps)), n_schunk, shots); block (32, kF4Warps).
// Each 8-lane strand runs kF4FRows rows of one 32-column side chunk.  Domain
// edges, CPML strips and padding columns are handled per cell; cells a step
// does not update keep their old values.
template <typename S>
__device__ __forceinline__ void f4_fwd_side_body(
    const TMGeom<float> &g, const F4Geom &q, const float *__restrict__ ca,
    const float *__restrict__ cb, const float *__restrict__ cq, const FwdState<float> &st0,
    S *__restrict__ est, S *__restrict__ cst, const PointCSR &src, const PointCSR &rec,
    const unsigned char *rowf, const float *__restrict__ f_t, float *__restrict__ r_t, int bx,
    int cy) {
  constexpr int RS = kF4FRows;
  const int seg = (bx * kF4Warps + threadIdx.y) * 4 + (threadIdx.x >> 3);
  if (seg >= q.n_sseg) return;
  const int y0 = seg * RS, yend = min(y0 + RS, g.ny);
  const int chunk = cy < q.n_lchunk ? cy : q.r_chunk0 + (cy - q.n_lchunk);
  const int jx = chunk * 32 + (threadIdx.x & 7) * 4;  // pitched column of the group
  const int x = jx - q.padl;                           // caller column
  const int nx = g.nx, ny = g.ny;
  if (x + 3 < 0 || x >= nx) return;
  if (x >= q.xl && x < q.xr) return;  // column band (other kernels)
  const int s = blockIdx.z;
  const int64_t base = (int64_t)s * q.pshot;
  const FwdState<float> st = shot_state(st0, base);
  if (g.ca_b) ca += base;
  if (g.cb_b) cb += base;
  if (g.cq_b) cq += base;
  const int64_t cbase = (int64_t)s * g.N;
  const int pitch = q.pitch;
  const float rdy = g.rdy, rdx = g.rdx;
  const int lo = max(0, -x), hi = min(4, nx - x);  // valid cells of the group

  bool xe[4], xhz[4], xsh[4], xse[4];
  bool lane_sh = false, lane_se = false;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int xc = x + k;
    xe[k] = xc >= 1 && xc < nx;       // E and H-x columns
    xhz[k] = xc >= 1 && xc < nx - 1;  // H-z columns
    xsh[k] = xhz[k] && (xc < g.pml_x0 || xc >= g.pml_x1h);
    xse[k] = xe[k] && (xc < g.pml_x0 || xc >= g.pml_x1);
    lane_sh = lane_sh || xsh[k];
    lane_se = lane_se || xse[k];
  }
  const int xl = x - 1;
  const bool xhzl = xl >= 1 && xl < nx - 1;
  const bool xshl = xhzl && (xl < g.pml_x0 || xl >= g.pml_x1h);
  lane_sh = lane_sh || xshl;
  const V4 zero{{0.f, 0.f, 0.f, 0.f}};
  // x profiles of the strip columns (1 and 0 elsewhere), read once
  float pxb[4], pxa[4], pxk[4], peb[4], pea[4], pek[4], plb = 0.f, pla = 0.f, plk = 1.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    pxb[k] = xsh[k] ? __ldg(g.bxh + x + k) : 0.f;
    pxa[k] = xsh[k] ? __ldg(g.axh + x + k) : 0.f;
    pxk[k] = xsh[k] ? __ldg(g.kxh + x + k) : 1.f;
    peb[k] = xse[k] ? __ldg(g.bx + x + k) : 0.f;
    pea[k] = xse[k] ? __ldg(g.ax + x + k) : 0.f;
    pek[k] = xse[k] ? __ldg(g.kx + x + k) : 1.f;
  }
  if (xshl) {
    plb = __ldg(g.bxh + xl);
    pla = __ldg(g.axh + xl);
    plk = __ldg(g.kxh + xl);
  }

  // Prologue: Ey(y0) and the new H-x of row y0-1.
  int j = (y0 - 1) * pitch + jx;
  V4 e0 = ldv(st.ey + j + pitch), hxp;
  {
    const int y = y0 - 1;
    const V4 em = ldv(st.ey + j), h = ldv(st.hx + j), c = ldv(cq + j);
    hxp = h;
    if (y >= 1 && y < ny - 1) {
      const bool zs = y < g.pml_y0 || y >= g.pml_y1h;
      V4 d;
#pragma unroll
      for (int k = 0; k < 4; ++k) d.c[k] = (e0.c[k] - em.c[k]) * rdy;
      if (zs) {
        const V4 mz = ldv(st.mez + j);
        const float zb = __ldg(g.byh + y), za = __ldg(g.ayh + y), zk = __ldg(g.kyh + y);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float m = zb * mz.c[k] + za * d.c[k];
          d.c[k] = div_k(d.c[k], zk) + m;
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) hxp.c[k] = sel(xe[k], h.c[k] - c.c[k] * d.c[k], h.c[k]);
    }
  }
  j += pitch;
#pragma unroll
  for (int r = 0; r < RS; ++r) {
    const int y = y0 + r;
    if (y >= yend) break;
    const bool hxu = y >= 1 && y < ny - 1;
    const bool zs = hxu && (y < g.pml_y0 || y >= g.pml_y1h);
    const bool yh = y >= 1;
    const bool ys = yh && (y < g.pml_y0 || y >= g.pml_y1);
    const bool lsh = yh && lane_sh, lse = yh && lane_se;
    // ---- loads
    const V4 e1 = ldv(st.ey + j + pitch), hx = ldv(st.hx + j), hz = ldv(st.hz + j);
    const V4 c = ldv(cq + j), a = ldv(ca + j), b = ldv(cb + j);
    const float er = __ldg(st.ey + j + 4), el = __ldg(st.ey + j - 1);
    const float hzl = __ldg(st.hz + j - 1), cql = __ldg(cq + j - 1);
    const V4 mez = zs ? ldv(st.mez + j) : zero;
    const V4 mex = lsh ? ldv(st.mex + j) : zero;
    const float mexl = (yh && xshl) ? __ldg(st.mex + j - 1) : 0.f;
    const V4 mhz = lse ? ldv_rw(st.mhz + j) : zero;
    const V4 mhx = ys ? ldv_rw(st.mhx + j) : zero;
    // ---- H-x (row y)
    V4 hxn = hx;
    if (hxu) {
      V4 d;
#pragma unroll
      for (int k = 0; k < 4; ++k) d.c[k] = (e1.c[k] - e0.c[k]) * rdy;
      if (zs) {
        const float zb = __ldg(g.byh + y), za = __ldg(g.ayh + y), zk = __ldg(g.kyh + y);
        V4 mn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float m = zb * mez.c[k] + za * d.c[k];
          mn.c[k] = sel(xe[k], m, mez.c[k]);
          d.c[k] = div_k(d.c[k], zk) + m;
        }
        stv(st.mez_n + j, mn);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) hxn.c[k] = sel(xe[k], hx.c[k] - c.c[k] * d.c[k], hx.c[k]);
    }
    // ---- H-z (row y, columns x .. x+3 and x-1)
    V4 hzn = hz;
    float hznl = hzl;
    if (yh) {
      V4 d;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float erk = k < 3 ? e0.c[k < 3 ? k + 1 : 3] : er;
        d.c[k] = (erk - e0.c[k]) * rdx;
      }
      float dl = (e0.c[0] - el) * rdx;
      if (lane_sh) {
        V4 mn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float m = pxb[k] * mex.c[k] + pxa[k] * d.c[k];
          mn.c[k] = sel(xsh[k], m, mex.c[k]);
          d.c[k] = sel(xsh[k], div_k(d.c[k], pxk[k]) + m, d.c[k]);
        }
        const float ml = plb * mexl + pla * dl;
        dl = sel(xshl, div_k(dl, plk) + ml, dl);
        stv(st.mex_n + j, mn);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) hzn.c[k] = sel(xhz[k], hz.c[k] + c.c[k] * d.c[k], hz.c[k]);
      hznl = sel(xhzl, hzl + cql * dl, hzl);
    }
    stv(st.hx_n + j, hxn);
    stv(st.hz_n + j, hzn);
    // ---- E (row y)
    V4 en = e0;
    if (yh) {
      V4 dz, dy;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float left = k ? hzn.c[k ? k - 1 : 0] : hznl;
        dz.c[k] = (hzn.c[k] - left) * rdx;
        dy.c[k] = (hxn.c[k] - hxp.c[k]) * rdy;
      }
      if (lane_se) {
        V4 mn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float m = peb[k] * mhz.c[k] + pea[k] * dz.c[k];
          mn.c[k] = sel(xse[k], m, mhz.c[k]);
          dz.c[k] = sel(xse[k], div_k(dz.c[k], pek[k]) + m, dz.c[k]);
        }
        stv(st.mhz_n + j, mn);
      }
      if (ys) {
        const float yb = __ldg(g.by + y), ya = __ldg(g.ay + y), yk = __ldg(g.ky + y);
        V4 mn;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float m = yb * mhx.c[k] + ya * dy.c[k];
          mn.c[k] = sel(xe[k], m, mhx.c[k]);
          dy.c[k] = div_k(dy.c[k], yk) + m;
        }
        stv(st.mhx_n + j, mn);
      }
      const int64_t cell = cbase + (int64_t)y * nx + x;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float curl = dz.c[k] - dy.c[k];
        if (xe[k]) {
          if (est) store_stream(est + cell + k, Codec<S, float>::enc(e0.c[k]));
          if (cst) store_stream(cst + cell + k, Codec<S, float>::enc(curl));
        }
        en.c[k] = sel(xe[k], a.c[k] * e0.c[k] + b.c[k] * curl, e0.c[k]);
      }
    }
    const int tile = f4_tile(q, s, y, jx);
    const bool pts = f4_row_points(q, rowf, s, y) && !point_tile_empty(src, rec, tile);
    if (pts) points_add4(src, tile, y * nx + x, lo, hi, f_t, en);
    stv(st.ey_n + j, en);
    if (pts) points_rec4(rec, tile, y * nx + x, lo, hi, r_t, en);
    hxp = hxn;
    e0 = e1;
    j += pitch;
  }
}

// ---------------------------------------------------------------- kernels
template <typename S> struct F4Smem {
  S sb[kF4Warps][2][128];  // snapshot transpose buffers (Ey, curl H) per warp
};

// Blocks of one fused forward step (host-computed): [0, n_side) side,
// [n_side, n_side + n_band) band, then interior.  Side and band blocks come
// first so that their latency-bound work overlaps the bandwidth-bound
// interior.
struct F4Blocks {
  int side_x;        // side blocks per side chunk (row direction)
  int n_side, n_band, n_int;
};

// One forward time step in one launch.  Grid: (n_side + n_band + n_int, 1,
// shots); block (32, kF4Warps).  The register cap (5 blocks per SM) is the
// best measured trade-off between the interior's occupancy and the frame
// code's register needs.
template <typename S>
__global__ void __launch_bounds__(32 * kF4Warps, 5)
f4_fwd_step(TMGeom<float> g, F4Geom q, F4Blocks nb, const float *__restrict__ ca,
            const float *__restrict__ cb, const float *__restrict__ cq, FwdState<float> st,
            S *__restrict__ est, S *__restrict__ cst, PointCSR src, PointCSR rec,
            const unsigned char *__restrict__ rowf, const float *__restrict__ f_t,
            float *__restrict__ r_t) {
  __shared__ __align__(16) F4Smem<S> sm;
  int b = blockIdx.x;
  if (b < nb.n_side) {
    f4_fwd_side_body<S>(g, q, ca, cb, cq, st, est, cst, src, rec, rowf, f_t, r_t,
                        b % nb.side_x, b / nb.side_x);
    return;
  }
  b -= nb.n_side;
  S *sb_e = sm.sb[threadIdx.y][0], *sb_c = sm.sb[threadIdx.y][1];
  if (b < nb.n_band) {
    f4_fwd_cols_body<S, true>(g, q, ca, cb, cq, st, est, cst, src, rec, rowf, f_t, r_t,
                              b % q.n_ix, b / q.n_ix, sb_e, sb_c);
    return;
  }
  b -= nb.n_band;
  f4_fwd_cols_body<S, false>(g, q, ca, cb, cq, st, est, cst, src, rec, rowf, f_t, r_t,
                             b % q.n_ix, b / q.n_ix, sb_e, sb_c);
}

#ifndef __CUDACC_RTC__
// Host: decomposition of a grid for the fused kernels.
inline F4Geom f4_geom(const TMGeom<float> &g) {
  constexpr int RS = kF4Rows, FR = kF4FRows;
  F4Geom q{};
  int xl = g.pml_x0 + 1 > 2 ? g.pml_x0 + 1 : 2;
  int xr = g.pml_x1h < g.nx - 1 ? g.pml_x1h : g.nx - 1;
  int yt = g.pml_y0 + 1 > 2 ? g.pml_y0 + 1 : 2;
  int yb = g.pml_y1h < g.ny - 1 ? g.pml_y1h : g.ny - 1;
  const bool any = xr - xl >= 4 && yb - yt >= RS;
  if (any) {
    xr = xl + (xr - xl) / 4 * 4;
    yb = yt + (yb - yt) / RS * RS;
  } else {
    xl = xr = 0;
    yt = yb = g.ny;
  }
  q.padl = any ? (32 - xl % 32) % 32 : 0;
  q.pitch = (q.padl + g.nx + 31) / 32 * 32;
  q.pshot = (int64_t)g.ny * q.pitch;
  q.xl = xl;
  q.xr = xr;
  q.yt = yt;
  q.yb = yb;
  q.n_ix = any ? (xr - xl + 127) / 128 : 0;
  q.n_iseg = any ? (yb - yt) / RS : 0;
  q.n_btop = any ? (yt + RS - 1) / RS : 0;
  q.n_bbot = any ? (g.ny - yb + RS - 1) / RS : 0;
  q.n_chunks = q.pitch / 32;
  q.n_lchunk = any ? (xl + q.padl) / 32 : 0;
  q.r_chunk0 = any ? (xr + q.padl) / 32 : 0;
  q.n_schunk = q.n_lchunk + (q.n_chunks - q.r_chunk0);
  q.n_sseg = (g.ny + FR - 1) / FR;
  q.pt = PointTiles{q.n_chunks, (g.ny + kF4PtH - 1) / kF4PtH, kF4PtW, kF4PtH, q.padl};
  return q;
}
inline F4Blocks f4_blocks(const F4Geom &q) {
  F4Blocks b{};
  b.side_x = (q.n_sseg + 4 * kF4Warps - 1) / (4 * kF4Warps);
  b.n_side = q.n_schunk > 0 ? b.side_x * q.n_schunk : 0;
  b.n_band = q.n_ix * ((q.n_btop + q.n_bbot + kF4Warps - 1) / kF4Warps);
  b.n_int = q.n_ix * ((q.n_iseg + kF4Warps - 1) / kF4Warps);
  return b;
}
#endif

}  // namespace tb
