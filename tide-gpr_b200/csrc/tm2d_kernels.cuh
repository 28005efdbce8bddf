// Device kernels for the TM2D time-stepping path on sm_100a.
//
// Field layout is the reference's: every field and CPML memory is a
// contiguous [n_shots, ny, nx] array of T; coefficients are [ny, nx] (or
// [n_shots, ny, nx] when batched); CPML profiles are 1-D.  All geometry is
// passed by value in TMGeom so kernels are re-entrant.
//
// Numerics: every expression keeps the reference's operation order and the
// translation unit is compiled with --fmad=false and IEEE division, so the
// forward reproduces the reference CPU backend bit for bit
// (src/tide/csrc/tm2d/maxwell_tm_core.cuh:448-599) and the adjoint
// reproduces the exact transpose of src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:954-1165.
//
// Sources and receivers are not separate launches.  A per-call setup builds,
// for each CTA tile (32 columns x tile_h rows) of each shot, the list of point entries that fall in it
// (CSR by tile, entries in ascending entry order).  The E-update kernel (and
// the adjoint H-update kernel) then finishes each cell in registers: it adds
// the source terms of its cell in entry order, writes the cell once, and
// records the receivers of its cell.  This reproduces the reference's
// add_sources_ey -> record_receivers_ey sequence (maxwell.cu:89-141) without
// two extra launches per step.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace tb {

constexpr int kTileX = 32;  // CTA tile width of the cell kernels (x fastest)

// Staggered-grid coefficients (src/tide/csrc/common/staggered_grid.h:229-417).
template <int ST> struct FD;
template <> struct FD<2> {
  static constexpr int P = 1;
  __device__ static constexpr double c(int) { return 1.0; }
};
template <> struct FD<4> {
  static constexpr int P = 2;
  __device__ static constexpr double c(int m) {
    return m == 0 ? 9.0 / 8.0 : -1.0 / 24.0;
  }
};
template <> struct FD<6> {
  static constexpr int P = 3;
  __device__ static constexpr double c(int m) {
    return m == 0 ? 75.0 / 64.0 : (m == 1 ? -25.0 / 384.0 : 3.0 / 640.0);
  }
};
template <> struct FD<8> {
  static constexpr int P = 4;
  __device__ static constexpr double c(int m) {
    return m == 0   ? 1225.0 / 1024.0
           : m == 1 ? -245.0 / 3072.0
           : m == 2 ? 49.0 / 5120.0
                    : -5.0 / 7168.0;
  }
};

// Step-indexed pointers of a launch replayed from a captured block of time
// steps.  The captured launch holds the pointers of the block it was
// captured for; replay j (the device word *blk, advanced by the block's last
// launch) moves each of them by j times its per-block advance, in elements.
// blk == nullptr: an ordinary launch whose pointers are used as given.
struct StepShift {
  const int64_t *blk = nullptr;
  int64_t src = 0;   // source amplitudes (forward) / their gradient (adjoint)
  int64_t rec = 0;   // receiver records (forward) / their gradient (adjoint)
  int64_t snap = 0;  // snapshot slots
  int64_t hist = 0;  // slots of a stored history the step reads (Born tangent)
  __device__ __forceinline__ int64_t block() const { return blk ? *blk : 0; }
};
template <typename P>
__device__ __forceinline__ P *shifted(P *p, int64_t adv, int64_t j) {
  return (p && j) ? p + adv * j : p;
}

template <typename T> struct TMGeom {
  const T *ay, *by, *ayh, *byh, *ax, *bx, *axh, *bxh;
  const T *ky, *kyh, *kx, *kxh;
  T rdy, rdx;
  int ny, nx;
  int64_t N;  // ny * nx
  int n_shots;
  int pml_y0, pml_y1, pml_x0, pml_x1;
  int pml_y1h, pml_x1h;  // half-grid inner edges (maxwell_tm_core.cuh:458-463)
  bool ca_b, cb_b, cq_b;
};

// CSR of point entries by (shot, tile).  start has n_tiles + 1 entries.
struct PointCSR {
  const int *start;  // nullptr when the list is empty
  const int *cell;   // flat cell index within the shot
  const int *ent;    // entry index e = shot * n_per_shot + k
};

__device__ int g_tide_dev_err;  // device-side error word (see tide_b200_device_status)

template <typename T> __device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// Forward staggered differences (maxwell_tm_core.cuh:64-190), generic in the
// stencil order.  For order 2 the unit coefficient multiply is exact.
template <typename T, int ST>
__device__ __forceinline__ T d_y1(const T *f, int64_t i, int nx, T rd) {
  T acc = (T)FD<ST>::c(0) * (ldg(f + i) - ldg(f + i - nx));
#pragma unroll
  for (int m = 1; m < FD<ST>::P; ++m)
    acc = acc + (T)FD<ST>::c(m) * (ldg(f + i + (int64_t)m * nx) - ldg(f + i - (int64_t)(m + 1) * nx));
  return acc * rd;
}
template <typename T, int ST>
__device__ __forceinline__ T d_x1(const T *f, int64_t i, T rd) {
  T acc = (T)FD<ST>::c(0) * (ldg(f + i) - ldg(f + i - 1));
#pragma unroll
  for (int m = 1; m < FD<ST>::P; ++m)
    acc = acc + (T)FD<ST>::c(m) * (ldg(f + i + m) - ldg(f + i - (m + 1)));
  return acc * rd;
}
template <typename T, int ST>
__device__ __forceinline__ T d_yh1(const T *f, int64_t i, int nx, T rd) {
  T acc = (T)FD<ST>::c(0) * (ldg(f + i + nx) - ldg(f + i));
#pragma unroll
  for (int m = 1; m < FD<ST>::P; ++m)
    acc = acc + (T)FD<ST>::c(m) * (ldg(f + i + (int64_t)(m + 1) * nx) - ldg(f + i - (int64_t)m * nx));
  return acc * rd;
}
template <typename T, int ST>
__device__ __forceinline__ T d_xh1(const T *f, int64_t i, T rd) {
  T acc = (T)FD<ST>::c(0) * (ldg(f + i + 1) - ldg(f + i));
#pragma unroll
  for (int m = 1; m < FD<ST>::P; ++m)
    acc = acc + (T)FD<ST>::c(m) * (ldg(f + i + m + 1) - ldg(f + i - m));
  return acc * rd;
}

// Snapshot codecs: identity for T, round-to-nearest-even for bf16.
template <typename S, typename T> struct Codec {
  __device__ static __forceinline__ S enc(T v) { return (S)v; }
  __device__ static __forceinline__ T dec(S v) { return (T)v; }
};
template <typename T> struct Codec<__nv_bfloat16, T> {
  __device__ static __forceinline__ __nv_bfloat16 enc(T v) { return __float2bfloat16((float)v); }
  __device__ static __forceinline__ T dec(__nv_bfloat16 v) { return (T)__bfloat162float(v); }
};

// Accumulate (in entry order) the values of all point entries at `cell` of
// tile `tile`: acc = acc + v[e] for each entry e at the cell.
template <typename T>
__device__ __forceinline__ T point_accumulate(const PointCSR &pl, int tile, int cell,
                                              const T *vals, T acc) {
  if (pl.start == nullptr || vals == nullptr) return acc;
  const int b = __ldg(pl.start + tile), e = __ldg(pl.start + tile + 1);
  for (int k = b; k < e; ++k)
    if (__ldg(pl.cell + k) == cell) acc = acc + ldg(vals + __ldg(pl.ent + k));
  return acc;
}
template <typename T>
__device__ __forceinline__ void point_record(const PointCSR &pl, int tile, int cell, T *out,
                                             T v) {
  if (pl.start == nullptr || out == nullptr) return;
  const int b = __ldg(pl.start + tile), e = __ldg(pl.start + tile + 1);
  for (int k = b; k < e; ++k)
    if (__ldg(pl.cell + k) == cell) out[__ldg(pl.ent + k)] = v;
}
__device__ __forceinline__ bool point_tile_empty(const PointCSR &a, const PointCSR &b, int tile) {
  bool ea = a.start == nullptr || __ldg(a.start + tile) == __ldg(a.start + tile + 1);
  bool eb = b.start == nullptr || __ldg(b.start + tile) == __ldg(b.start + tile + 1);
  return ea && eb;
}

// ---------------------------------------------------------------------------
// Launch shape shared by the stencil kernels: blocks of 32 (x) x 8 (y)
// threads; each thread owns one column x and R consecutive rows, so a warp
// touches 32 consecutive floats of R rows and every thread issues all of its
// loads before any arithmetic (memory-level parallelism is what bounds these
// kernels; one cell per thread left the SMs waiting on L1/L2).
constexpr int kBlockY = 8;

// ---------------------------------------------------------------------------
// Interior fast paths (stencil order 2).  A CTA whose cells and stencil
// neighbours all lie outside the CPML strips (and so away from the domain
// edges) needs none of the strip logic; most of the grid is such tiles.  They
// take a branch-free path: 32-bit offsets from the shot's base pointer,
// x-neighbours exchanged with warp shuffles (blockDim.x == 32, so threadIdx.x
// is the lane), y-neighbours reused from registers.  Every value is computed
// with the same operations in the same order as the general path, so both
// paths give bit-identical results.  Offsets fit in int32: the host rejects
// grids with ny * nx >= 2^31.
constexpr unsigned kFull = 0xffffffffu;

template <typename T, int R>
__device__ __forceinline__ void fwd_h_fast(const TMGeom<T> &g, const T *__restrict__ cq,
                                           const T *__restrict__ ey, T *__restrict__ hx,
                                           T *__restrict__ hz, int x, int y0) {
  const int nx = g.nx, j0 = y0 * nx + x;
  T e[R + 1], c[R], vx[R], vz[R], er[R];
#pragma unroll
  for (int r = 0; r <= R; ++r) e[r] = ldg(ey + j0 + r * nx);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    c[r] = ldg(cq + j0 + r * nx);
    vx[r] = hx[j0 + r * nx];
    vz[r] = hz[j0 + r * nx];
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    er[r] = __shfl_down_sync(kFull, e[r], 1);
    if (threadIdx.x == 31) er[r] = ldg(ey + j0 + r * nx + 1);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const T dz = (e[r + 1] - e[r]) * g.rdy;
    const T dx = (er[r] - e[r]) * g.rdx;
    hx[j0 + r * nx] = vx[r] - c[r] * dz;
    hz[j0 + r * nx] = vz[r] + c[r] * dx;
  }
}

// Forward H half-step (maxwell_tm_core.cuh:448-502).  Grid: x over the update
// domain [P, nx-P+1), y over row groups, z = shot.
template <typename T, int ST, int R>
__global__ void __launch_bounds__(256)
k_fwd_h(TMGeom<T> g, const T *__restrict__ cq, const T *__restrict__ ey, T *__restrict__ hx,
        T *__restrict__ hz, T *__restrict__ m_ey_x, T *__restrict__ m_ey_z) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x + P;
  const int y0 = (blockIdx.y * kBlockY + threadIdx.y) * R + P;
  const int64_t base = (int64_t)blockIdx.z * g.N;
  if constexpr (ST == 2) {
    // Interior tile: no strip cell for Hx or Hz (block-uniform test).
    const int tx0 = blockIdx.x * kTileX + P, ty0 = blockIdx.y * kBlockY * R + P;
    if (tx0 >= g.pml_x0 && tx0 + kTileX <= g.pml_x1h && ty0 >= g.pml_y0 &&
        ty0 + kBlockY * R <= g.pml_y1h) {
      fwd_h_fast<T, R>(g, g.cq_b ? cq + base : cq, ey + base, hx + base, hz + base, x, y0);
      return;
    }
  }
  const int ye = g.ny - P + 1;
  if (x >= g.nx - P + 1 || y0 >= ye) return;
  const bool do_hz = x < g.nx - P;
  const bool px = x < g.pml_x0 || x >= g.pml_x1h;
  T cqv[R], dz[R], dx[R], hxv[R], hzv[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    if (y < ye) {
      const int64_t j = (int64_t)y * g.nx + x, i = base + j;
      cqv[r] = g.cq_b ? ldg(cq + i) : ldg(cq + j);
      if (y < g.ny - P) {
        dz[r] = d_yh1<T, ST>(ey, i, g.nx, g.rdy);
        hxv[r] = hx[i];
      }
      if (do_hz) {
        dx[r] = d_xh1<T, ST>(ey, i, g.rdx);
        hzv[r] = hz[i];
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    if (y >= ye) continue;
    const int64_t i = base + (int64_t)y * g.nx + x;
    if (y < g.ny - P) {
      T d = dz[r];
      if (y < g.pml_y0 || y >= g.pml_y1h) {
        const T m = ldg(g.byh + y) * m_ey_z[i] + ldg(g.ayh + y) * d;
        m_ey_z[i] = m;
        d = d / ldg(g.kyh + y) + m;
      }
      hx[i] = hxv[r] - cqv[r] * d;
    }
    if (do_hz) {
      T d = dx[r];
      if (px) {
        const T m = ldg(g.bxh + x) * m_ey_x[i] + ldg(g.axh + x) * d;
        m_ey_x[i] = m;
        d = d / ldg(g.kxh + x) + m;
      }
      hz[i] = hzv[r] + cqv[r] * d;
    }
  }
}

// Debye (1..n poles) state for the E kernel; n_poles == 0 disables it.
template <typename T> struct DebyeArgs {
  const T *a, *b, *cp;  // [n_poles, ny, nx]
  T *pol;               // [n_shots, n_poles, ny, nx]
  int n_poles;
  // snapshots of this step (element type S of the kernel), null: not recorded
  void *pol_st;   // P^t before the update, [n_shots, n_poles, ny, nx]
  void *esum_st;  // E^{t+1} + E^t, [n_shots, ny, nx]
};

template <typename S> __device__ __forceinline__ void store_stream(S *p, S v) { __stcs(p, v); }
template <> __device__ __forceinline__ void store_stream<__nv_bfloat16>(__nv_bfloat16 *p,
                                                                       __nv_bfloat16 v) {
  __stcs(reinterpret_cast<unsigned short *>(p), __bfloat16_as_ushort(v));
}
template <typename S> __device__ __forceinline__ S load_stream(const S *p) { return __ldcs(p); }
template <> __device__ __forceinline__ __nv_bfloat16 load_stream<__nv_bfloat16>(const __nv_bfloat16 *p) {
  return __ushort_as_bfloat16(__ldcs(reinterpret_cast<const unsigned short *>(p)));
}

// Forward E half-step, interior tile (no strip cell, no Debye); points of the
// tile are applied per cell exactly as in the general path.
template <typename T, typename S, int R>
__device__ __forceinline__ void fwd_e_fast(const TMGeom<T> &g, const T *__restrict__ ca,
                                           const T *__restrict__ cb, const T *__restrict__ hx,
                                           const T *__restrict__ hz, T *__restrict__ ey,
                                           S *__restrict__ est, S *__restrict__ cst, bool pts,
                                           const PointCSR &src, const PointCSR &rec, int tile,
                                           const T *__restrict__ f_t, T *__restrict__ r_t, int x,
                                           int y0) {
  const int nx = g.nx, j0 = y0 * nx + x;
  T vx[R + 1], vz[R], vzl[R], eo[R], a[R], b[R];
#pragma unroll
  for (int r = 0; r <= R; ++r) vx[r] = ldg(hx + j0 + (r - 1) * nx);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    vz[r] = ldg(hz + j0 + r * nx);
    eo[r] = ey[j0 + r * nx];
    a[r] = ldg(ca + j0 + r * nx);
    b[r] = ldg(cb + j0 + r * nx);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    vzl[r] = __shfl_up_sync(kFull, vz[r], 1);
    if (threadIdx.x == 0) vzl[r] = ldg(hz + j0 + r * nx - 1);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r * nx;
    const T dz = (vz[r] - vzl[r]) * g.rdx;
    const T dy = (vx[r + 1] - vx[r]) * g.rdy;
    const T curl = dz - dy;
    if (est) store_stream(est + j, Codec<S, T>::enc(eo[r]));
    if (cst) store_stream(cst + j, Codec<S, T>::enc(curl));
    T e = a[r] * eo[r] + b[r] * curl;
    if (pts) e = point_accumulate(src, tile, j, f_t, e);
    ey[j] = e;
    if (pts) point_record(rec, tile, j, r_t, e);
  }
}

// Forward E half-step with optional snapshot storage, Debye polarisation,
// source injection and receiver recording
// (maxwell_tm_core.cuh:504-599, maxwell_tm_cuda_inst.cu:382-457,
// maxwell.cu:89-141).  Grid covers the full [0,ny)x[0,nx) grid (tiles of 32 x
// 8R) so points outside the update domain are still injected and recorded.
template <typename T, int ST, typename S, int R, int BY = kBlockY>
__global__ void __launch_bounds__(32 * BY)
k_fwd_e(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cb, const T *__restrict__ hx,
        const T *__restrict__ hz, T *__restrict__ ey, T *__restrict__ m_hx_z,
        T *__restrict__ m_hz_x, S *__restrict__ ey_store, S *__restrict__ curl_store,
        DebyeArgs<T> db, PointCSR src, PointCSR rec, const T *__restrict__ f_t,
        T *__restrict__ r_t, StepShift sh) {
  constexpr int P = FD<ST>::P;
  if (sh.blk) {
    const int64_t jb = sh.block();
    f_t = shifted(f_t, sh.src, jb);
    r_t = shifted(r_t, sh.rec, jb);
    ey_store = shifted(ey_store, sh.snap, jb);
    curl_store = shifted(curl_store, sh.snap, jb);
  }
  const int x = blockIdx.x * kTileX + threadIdx.x;
  const int y0 = (blockIdx.y * BY + threadIdx.y) * R;
  const int s = blockIdx.z;
  const int tile = (s * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const bool pts = !point_tile_empty(src, rec, tile);
  const int64_t base = (int64_t)s * g.N;
  if constexpr (ST == 2) {
    const int tx0 = blockIdx.x * kTileX, ty0 = blockIdx.y * BY * R;
    if (db.n_poles == 0 && tx0 >= g.pml_x0 && tx0 + kTileX <= g.pml_x1 && ty0 >= g.pml_y0 &&
        ty0 + BY * R <= g.pml_y1) {
      fwd_e_fast<T, S, R>(g, g.ca_b ? ca + base : ca, g.cb_b ? cb + base : cb, hx + base,
                          hz + base, ey + base, ey_store ? ey_store + base : nullptr,
                          curl_store ? curl_store + base : nullptr, pts, src, rec, tile, f_t,
                          r_t, x, y0);
      return;
    }
  }
  if (x >= g.nx || y0 >= g.ny) return;
  const bool xdom = x >= P && x < g.nx - P + 1;
  const bool px = x < g.pml_x0 || x >= g.pml_x1;
  T eo[R], en[R], dhz[R], dhx[R], cav[R], cbv[R];
  bool dom[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    dom[r] = xdom && y >= P && y < g.ny - P + 1;
    if (dom[r] || (pts && y < g.ny)) {
      const int64_t j = (int64_t)y * g.nx + x, i = base + j;
      eo[r] = ey[i];
      if (dom[r]) {
        cav[r] = g.ca_b ? ldg(ca + i) : ldg(ca + j);
        cbv[r] = g.cb_b ? ldg(cb + i) : ldg(cb + j);
        dhz[r] = d_x1<T, ST>(hz, i, g.rdx);
        dhx[r] = d_y1<T, ST>(hx, i, g.nx, g.rdy);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    if (!(dom[r] || (pts && y < g.ny))) continue;
    const int64_t j = (int64_t)y * g.nx + x, i = base + j;
    T e = eo[r];
    if (dom[r]) {
      T dz = dhz[r], dy = dhx[r];
      if (px) {
        const T m = ldg(g.bx + x) * m_hz_x[i] + ldg(g.ax + x) * dz;
        m_hz_x[i] = m;
        dz = dz / ldg(g.kx + x) + m;
      }
      if (y < g.pml_y0 || y >= g.pml_y1) {
        const T m = ldg(g.by + y) * m_hx_z[i] + ldg(g.ay + y) * dy;
        m_hx_z[i] = m;
        dy = dy / ldg(g.ky + y) + m;
      }
      const T curl = dz - dy;
      if (ey_store) store_stream(ey_store + i, Codec<S, T>::enc(e));
      if (curl_store) store_stream(curl_store + i, Codec<S, T>::enc(curl));
      e = cav[r] * e + cbv[r] * curl;
      if (db.n_poles > 0) {
        T pol_term = (T)0;
        for (int p = 0; p < db.n_poles; ++p) {
          const int64_t pi = ((int64_t)s * db.n_poles + p) * g.N + j;
          const T pv = db.pol[pi];
          if (db.pol_st) store_stream(static_cast<S *>(db.pol_st) + pi, Codec<S, T>::enc(pv));
          pol_term = pol_term + ldg(db.cp + (int64_t)p * g.N + j) * pv;
        }
        e = e + pol_term;
      }
    }
    if (pts) e = point_accumulate(src, tile, (int)j, f_t, e);
    ey[i] = e;
    if (dom[r] && db.n_poles > 0) {
      const T e_sum = e + eo[r];
      if (db.esum_st) store_stream(static_cast<S *>(db.esum_st) + i, Codec<S, T>::enc(e_sum));
      for (int p = 0; p < db.n_poles; ++p) {
        const int64_t c = (int64_t)p * g.N + j;
        const int64_t pi = ((int64_t)s * db.n_poles + p) * g.N + j;
        db.pol[pi] = ldg(db.a + c) * db.pol[pi] + ldg(db.b + c) * e_sum;
      }
    }
    if (pts) point_record(rec, tile, (int)j, r_t, e);
    en[r] = e;
  }
  (void)en;
}

// ---------------------------------------------------------------------------
// Exact adjoint, E-phase (maxwell_tm_cuda_inst.cu:954-1027).  The CPML memory
// adjoints ping-pong between m (current, read) and m_n (next, written); the
// next buffers are written only in their strips because both buffers hold
// zeros elsewhere for the whole call (cleared on entry).
template <typename T, int ST>
__device__ __forceinline__ T raw_x(const TMGeom<T> &g, const T *cb, const T *lam, const T *m,
                                   int64_t base, int y, int x) {
  constexpr int P = FD<ST>::P;
  if (y < P || y >= g.ny - P + 1 || x < P || x >= g.nx - P + 1) return (T)0;
  const int64_t j = (int64_t)y * g.nx + x, i = base + j;
  const T q = (g.cb_b ? ldg(cb + i) : ldg(cb + j)) * ldg(lam + i);
  if (x >= g.pml_x0 && x < g.pml_x1) return q;
  const T mn = ldg(g.bx + x) * ldg(m + i) + q;
  return ldg(g.ax + x) * mn + q / ldg(g.kx + x);
}
template <typename T, int ST>
__device__ __forceinline__ T raw_y(const TMGeom<T> &g, const T *cb, const T *lam, const T *m,
                                   int64_t base, int y, int x) {
  constexpr int P = FD<ST>::P;
  if (y < P || y >= g.ny - P + 1 || x < P || x >= g.nx - P + 1) return (T)0;
  const int64_t j = (int64_t)y * g.nx + x, i = base + j;
  const T q = (g.cb_b ? ldg(cb + i) : ldg(cb + j)) * ldg(lam + i);
  if (y >= g.pml_y0 && y < g.pml_y1) return -q;
  const T mn = ldg(g.by + y) * ldg(m + i) - q;
  return ldg(g.ay + y) * mn - q / ldg(g.ky + y);
}

// Adjoint E-phase, interior tile: raw_x = q and raw_y = -q with q = cb * lam,
// no memory adjoint in the strips of these cells or their neighbours.
template <typename T, int R>
__device__ __forceinline__ void adj_e_fast(const TMGeom<T> &g, const T *__restrict__ cb,
                                           const T *__restrict__ lam, T *__restrict__ lhx,
                                           T *__restrict__ lhz, int x, int y0) {
  const int nx = g.nx, j0 = y0 * nx + x;
  T q[R + 1], qr[R], vx[R], vz[R];
#pragma unroll
  for (int r = 0; r <= R; ++r) q[r] = ldg(cb + j0 + r * nx) * ldg(lam + j0 + r * nx);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    vx[r] = lhx[j0 + r * nx];
    vz[r] = lhz[j0 + r * nx];
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    qr[r] = __shfl_down_sync(kFull, q[r], 1);
    if (threadIdx.x == 31) qr[r] = ldg(cb + j0 + r * nx + 1) * ldg(lam + j0 + r * nx + 1);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const T ax_ = (T)1 * (q[r] - qr[r]);
    lhz[j0 + r * nx] = vz[r] + ax_ * g.rdx;
    const T ay_ = (T)1 * ((-q[r]) - (-q[r + 1]));
    lhx[j0 + r * nx] = vx[r] + ay_ * g.rdy;
  }
}

template <typename T, int ST, int R, int BY = kBlockY>
__global__ void __launch_bounds__(32 * BY)
k_adj_e(TMGeom<T> g, const T *__restrict__ cb, const T *__restrict__ lam_ey,
        T *__restrict__ lam_hx, T *__restrict__ lam_hz, const T *__restrict__ m_hx_z,
        const T *__restrict__ m_hz_x, T *__restrict__ m_hx_z_n, T *__restrict__ m_hz_x_n) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x + P;
  const int y0 = (blockIdx.y * BY + threadIdx.y) * R + P;
  const int64_t base = (int64_t)blockIdx.z * g.N;
  if constexpr (ST == 2) {
    // Interior tile: cells and their +1 neighbours outside the strips.
    const int tx0 = blockIdx.x * kTileX + P, ty0 = blockIdx.y * BY * R + P;
    if (tx0 >= g.pml_x0 && tx0 + kTileX < g.pml_x1 && ty0 >= g.pml_y0 &&
        ty0 + BY * R < g.pml_y1) {
      adj_e_fast<T, R>(g, g.cb_b ? cb + base : cb, lam_ey + base, lam_hx + base, lam_hz + base,
                       x, y0);
      return;
    }
  }
  const int ye = g.ny - P + 1;
  if (x >= g.nx - P + 1 || y0 >= ye) return;
  const bool px = x < g.pml_x0 || x >= g.pml_x1;
  // raw_y on rows y0-P+1 .. y0+R-1+P, raw_x on columns x-P+1 .. x+P per row.
  T ry[R + 2 * P - 1];
#pragma unroll
  for (int k = 0; k < R + 2 * P - 1; ++k)
    ry[k] = raw_y<T, ST>(g, cb, lam_ey, m_hx_z, base, y0 - P + 1 + k, x);
  T rx[R][2 * P];
  T lhx[R], lhz[R], qv[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
#pragma unroll
    for (int k = 0; k < 2 * P; ++k) rx[r][k] = raw_x<T, ST>(g, cb, lam_ey, m_hz_x, base, y, x - P + 1 + k);
    if (y < ye) {
      const int64_t j = (int64_t)y * g.nx + x, i = base + j;
      qv[r] = (g.cb_b ? ldg(cb + i) : ldg(cb + j)) * ldg(lam_ey + i);
      lhx[r] = lam_hx[i];
      lhz[r] = lam_hz[i];
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    if (y >= ye) continue;
    const int64_t i = base + (int64_t)y * g.nx + x;
    if (px) m_hz_x_n[i] = ldg(g.bx + x) * ldg(m_hz_x + i) + qv[r];
    if (y < g.pml_y0 || y >= g.pml_y1) m_hx_z_n[i] = ldg(g.by + y) * ldg(m_hx_z + i) - qv[r];
    // diff_x1_adj: sum_m c_m (raw(x-m) - raw(x+1+m)); rx[r][k] holds raw(x-P+1+k)
    T ax_ = (T)FD<ST>::c(0) * (rx[r][P - 1] - rx[r][P]);
#pragma unroll
    for (int m = 1; m < P; ++m) ax_ = ax_ + (T)FD<ST>::c(m) * (rx[r][P - 1 - m] - rx[r][P + m]);
    lam_hz[i] = lhz[r] + ax_ * g.rdx;
    // diff_y1_adj: sum_m c_m (raw(y-m) - raw(y+1+m)); ry[k] holds raw(y0-P+1+k)
    T ay_ = (T)FD<ST>::c(0) * (ry[r + P - 1] - ry[r + P]);
#pragma unroll
    for (int m = 1; m < P; ++m) ay_ = ay_ + (T)FD<ST>::c(m) * (ry[r + P - 1 - m] - ry[r + P + m]);
    lam_hx[i] = lhx[r] + ay_ * g.rdy;
  }
}

// ---------------------------------------------------------------------------
// Exact adjoint, H-phase (maxwell_tm_cuda_inst.cu:1082-1165), fused with the
// adjoint-source injection at receivers, the source-gradient recording
// (maxwell.cu:107-161) and the coefficient gradient of this step
// (maxwell_tm_cuda_inst.cu:834-871): the final adjoint of step t is in a
// register when the cell is written, so grad_ca += lam * Ey^t * k and
// grad_cb += lam * curlH^t * k are taken there.  Each thread loops over all
// shots of the call and sums their image terms before one read-modify-write
// of the model-shaped gradient (batched models keep one gradient per shot).
template <typename T, int ST>
__device__ __forceinline__ T raw_eyz(const TMGeom<T> &g, const T *cq, const T *lhx, const T *m,
                                     int64_t base, int y, int x) {
  constexpr int P = FD<ST>::P;
  if (y < P || y >= g.ny - P || x < P || x >= g.nx - P + 1) return (T)0;
  const int64_t j = (int64_t)y * g.nx + x, i = base + j;
  const T adj = -(g.cq_b ? ldg(cq + i) : ldg(cq + j)) * ldg(lhx + i);
  if (y >= g.pml_y0 && y < g.pml_y1h) return adj;
  const T mn = ldg(g.byh + y) * ldg(m + i) + adj;
  return ldg(g.ayh + y) * mn + adj / ldg(g.kyh + y);
}
template <typename T, int ST>
__device__ __forceinline__ T raw_eyx(const TMGeom<T> &g, const T *cq, const T *lhz, const T *m,
                                     int64_t base, int y, int x) {
  constexpr int P = FD<ST>::P;
  if (y < P || y >= g.ny - P + 1 || x < P || x >= g.nx - P) return (T)0;
  const int64_t j = (int64_t)y * g.nx + x, i = base + j;
  const T adj = (g.cq_b ? ldg(cq + i) : ldg(cq + j)) * ldg(lhz + i);
  if (x >= g.pml_x0 && x < g.pml_x1h) return adj;
  const T mn = ldg(g.bxh + x) * ldg(m + i) + adj;
  return ldg(g.axh + x) * mn + adj / ldg(g.kxh + x);
}

template <typename T, typename S> struct GradArgs {
  const S *ey_st;  // snapshot Ey^t of the step being imaged (nullptr: skip)
  const S *cu_st;  // snapshot curl H^t
  T *grad_ca;      // [ny, nx], or [n_shots, ny, nx] when `batched`
  T *grad_cb;
  T kscale;        // gradient sampling interval as T
  bool batched_ca, batched_cb;
  // Shots of the snapshot history: adjoint shot s images against snapshot
  // shot s % bg_shots (background_vjp_reuse); 0 = one snapshot per shot.
  int bg_shots = 0;
  __device__ __forceinline__ int64_t snap_base(int s, int64_t N) const {
    return (int64_t)(bg_shots > 0 ? s % bg_shots : s) * N;
  }
};

// Adjoint H-phase update of one cell (general path: strips, domain edges).
template <typename T, int ST>
__device__ __forceinline__ T adj_h_general(const TMGeom<T> &g, const T *__restrict__ ca,
                                           const T *__restrict__ cq,
                                           const T *__restrict__ lam_hx,
                                           const T *__restrict__ lam_hz,
                                           const T *__restrict__ m_ey_x,
                                           const T *__restrict__ m_ey_z, T *__restrict__ m_ey_x_n,
                                           T *__restrict__ m_ey_z_n, int64_t base, int y, int x,
                                           T lam) {
  constexpr int P = FD<ST>::P;
  const int64_t j = (int64_t)y * g.nx + x, i = base + j;
  const T cqs = g.cq_b ? ldg(cq + i) : ldg(cq + j);
  const T cas = g.ca_b ? ldg(ca + i) : ldg(ca + j);
  const bool py = y < g.pml_y0 || y >= g.pml_y1h;
  const bool px = x < g.pml_x0 || x >= g.pml_x1h;
  const T adj_y = -cqs * ldg(lam_hx + i);
  const T adj_x = cqs * ldg(lam_hz + i);
  if (y < g.ny - P && py) m_ey_z_n[i] = ldg(g.byh + y) * ldg(m_ey_z + i) + adj_y;
  if (x < g.nx - P && px) m_ey_x_n[i] = ldg(g.bxh + x) * ldg(m_ey_x + i) + adj_x;
  lam = cas * lam;
  T dz = (T)FD<ST>::c(0) * (raw_eyz<T, ST>(g, cq, lam_hx, m_ey_z, base, y - 1, x) -
                           raw_eyz<T, ST>(g, cq, lam_hx, m_ey_z, base, y, x));
#pragma unroll
  for (int m = 1; m < P; ++m)
    dz = dz + (T)FD<ST>::c(m) * (raw_eyz<T, ST>(g, cq, lam_hx, m_ey_z, base, y - 1 - m, x) -
                                 raw_eyz<T, ST>(g, cq, lam_hx, m_ey_z, base, y + m, x));
  T dx = (T)FD<ST>::c(0) * (raw_eyx<T, ST>(g, cq, lam_hz, m_ey_x, base, y, x - 1) -
                           raw_eyx<T, ST>(g, cq, lam_hz, m_ey_x, base, y, x));
#pragma unroll
  for (int m = 1; m < P; ++m)
    dx = dx + (T)FD<ST>::c(m) * (raw_eyx<T, ST>(g, cq, lam_hz, m_ey_x, base, y, x - 1 - m) -
                                 raw_eyx<T, ST>(g, cq, lam_hz, m_ey_x, base, y, x + m));
  return lam + (dz * g.rdy + dx * g.rdx);
}

// Adjoint H-phase, interior tile (stencil 2): raw_eyz = -cq * lam_hx and
// raw_eyx = cq * lam_hz for the cells and their -1 neighbours.
template <typename T, int R>
__device__ __forceinline__ void adj_h_fast(const TMGeom<T> &g, const T *__restrict__ ca,
                                           const T *__restrict__ cq,
                                           const T *__restrict__ lhx,
                                           const T *__restrict__ lhz, const T *__restrict__ ley,
                                           int j0, T (&lam)[R]) {
  const int nx = g.nx;
  T rz[R + 1], rx[R], rxl[R], a[R];
#pragma unroll
  for (int r = 0; r <= R; ++r) {
    const int j = j0 + (r - 1) * nx;
    rz[r] = -ldg(cq + j) * ldg(lhx + j);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r * nx;
    rx[r] = ldg(cq + j) * ldg(lhz + j);
    a[r] = ldg(ca + j);
    lam[r] = ley[j];
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    rxl[r] = __shfl_up_sync(kFull, rx[r], 1);
    if (threadIdx.x == 0) rxl[r] = ldg(cq + j0 + r * nx - 1) * ldg(lhz + j0 + r * nx - 1);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const T dz = (T)1 * (rz[r] - rz[r + 1]);
    const T dx = (T)1 * (rxl[r] - rx[r]);
    lam[r] = a[r] * lam[r];
    lam[r] = lam[r] + (dz * g.rdy + dx * g.rdx);
  }
}

template <typename T, int ST, typename S, int R>
__global__ void __launch_bounds__(256)
k_adj_h(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cq,
        const T *__restrict__ lam_hx, const T *__restrict__ lam_hz, T *__restrict__ lam_ey,
        const T *__restrict__ m_ey_x, const T *__restrict__ m_ey_z, T *__restrict__ m_ey_x_n,
        T *__restrict__ m_ey_z_n, PointCSR rec, PointCSR src, const T *__restrict__ gr_t,
        T *__restrict__ gf_t, GradArgs<T, S> ga, StepShift sh) {
  constexpr int P = FD<ST>::P;
  if (sh.blk) {
    const int64_t jb = sh.block();
    gr_t = shifted(gr_t, sh.rec, jb);
    gf_t = shifted(gf_t, sh.src, jb);
    ga.ey_st = shifted(ga.ey_st, sh.snap, jb);
    ga.cu_st = shifted(ga.cu_st, sh.snap, jb);
  }
  const int x = blockIdx.x * kTileX + threadIdx.x;
  const int y0 = (blockIdx.y * kBlockY + threadIdx.y) * R;
  const int tile_xy = blockIdx.y * gridDim.x + blockIdx.x;
  const int tiles_per_shot = gridDim.x * gridDim.y;
  bool fast = false;
  if constexpr (ST == 2) {
    // Interior tile: cells and their -1 neighbours outside the strips.
    const int tx0 = blockIdx.x * kTileX, ty0 = blockIdx.y * kBlockY * R;
    fast = !g.ca_b && !g.cq_b && tx0 - 1 >= g.pml_x0 && tx0 + kTileX <= g.pml_x1h &&
           ty0 - 1 >= g.pml_y0 && ty0 + kBlockY * R <= g.pml_y1h;
  }
  if (!fast && (x >= g.nx || y0 >= g.ny)) return;
  const bool imaging = ga.ey_st != nullptr || ga.cu_st != nullptr;
  T sum_ca[R], sum_cb[R];
#pragma unroll
  for (int r = 0; r < R; ++r) sum_ca[r] = sum_cb[r] = (T)0;
  const int j0 = y0 * g.nx + x;
  for (int s = 0; s < g.n_shots; ++s) {
    const int64_t base = (int64_t)s * g.N;
    const int64_t sbase = ga.snap_base(s, g.N);
    const int tile = s * tiles_per_shot + tile_xy;
    const bool pts = !point_tile_empty(src, rec, tile);
    T lam[R];
    bool live[R], dom[R];
    if (fast) {
      adj_h_fast<T, R>(g, ca, cq, lam_hx + base, lam_hz + base, lam_ey + base, j0, lam);
#pragma unroll
      for (int r = 0; r < R; ++r) live[r] = dom[r] = true;
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int y = y0 + r;
        dom[r] = x >= P && y >= P && x < g.nx - P + 1 && y < g.ny - P + 1;
        live[r] = y < g.ny && (dom[r] || pts);
        if (!live[r]) continue;
        lam[r] = lam_ey[base + (int64_t)y * g.nx + x];
        if (dom[r])
          lam[r] = adj_h_general<T, ST>(g, ca, cq, lam_hx, lam_hz, m_ey_x, m_ey_z, m_ey_x_n,
                                        m_ey_z_n, base, y, x, lam[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (!live[r]) continue;
      const int j = j0 + r * g.nx;
      const int64_t i = base + j;
      T v = lam[r];
      if (pts) v = point_accumulate(rec, tile, j, gr_t, v);
      lam_ey[i] = v;
      if (pts) point_record(src, tile, j, gf_t, v);
      if (imaging && dom[r]) {
        if (ga.ey_st) {
          const T t = v * Codec<S, T>::dec(load_stream(ga.ey_st + sbase + j)) * ga.kscale;
          if (ga.batched_ca) ga.grad_ca[i] = ga.grad_ca[i] + t;
          else sum_ca[r] = sum_ca[r] + t;
        }
        if (ga.cu_st) {
          const T t = v * Codec<S, T>::dec(load_stream(ga.cu_st + sbase + j)) * ga.kscale;
          if (ga.batched_cb) ga.grad_cb[i] = ga.grad_cb[i] + t;
          else sum_cb[r] = sum_cb[r] + t;
        }
      }
    }
  }
  if (!imaging) return;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    const bool dom = x >= P && y >= P && x < g.nx - P + 1 && y < g.ny - P + 1;
    if (!dom) continue;
    const int j = j0 + r * g.nx;
    if (ga.ey_st && !ga.batched_ca) ga.grad_ca[j] = ga.grad_ca[j] + sum_ca[r];
    if (ga.cu_st && !ga.batched_cb) ga.grad_cb[j] = ga.grad_cb[j] + sum_cb[r];
  }
}

// Clears a CPML memory array outside its absorbing strips along one axis
// (axis 0: rows [lo, hi) are cleared; axis 1: columns [lo, hi)).
template <typename T>
__global__ void k_zero_band(T *__restrict__ m, int n_shots, int ny, int nx, int axis, int lo,
                            int hi) {
  const int64_t n = (int64_t)n_shots * ny * nx;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = k % ((int64_t)ny * nx);
    const int v = axis == 0 ? (int)(c / nx) : (int)(c % nx);
    if (v >= lo && v < hi) m[k] = (T)0;
  }
}

// ---------------------------------------------------------------------------
// Point-list construction (once per call).  Entries with a negative index are
// skipped as in the reference; an index at or beyond ny*nx sets the device
// error word and is skipped instead of writing out of bounds.
// Tile of a cell: tiles of tile_w columns (counted from column -xoff) by
// tile_h rows, tiles_x x tiles_y per shot.
struct PointTiles {
  int tiles_x, tiles_y, tile_w, tile_h, xoff;
};
__device__ __forceinline__ int point_tile_of(int64_t idx, int s, int nx, const PointTiles &t) {
  const int y = (int)(idx / nx), x = (int)(idx % nx);
  return (s * t.tiles_y + y / t.tile_h) * t.tiles_x + (x + t.xoff) / t.tile_w;
}

__global__ void k_points_count(const int64_t *__restrict__ idx, int n_per_shot, int n_shots,
                               int64_t N, int nx, PointTiles pt, int *__restrict__ count) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_per_shot * n_shots) return;
  const int64_t v = idx[e];
  if (v < 0) return;
  if (v >= N) {
    atomicOr(&g_tide_dev_err, 1);
    return;
  }
  atomicAdd(count + point_tile_of(v, e / n_per_shot, nx, pt), 1);
}

// Per tile row i = shot * tiles_y + tile row: does any tile of the row hold a
// point of either list?  (start arrays are exclusive scans over the tiles.)
__global__ void k_points_rowflags(const int *__restrict__ s_start, const int *__restrict__ r_start,
                                  int tiles_x, int n_rows, unsigned char *__restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_rows) return;
  const int t0 = i * tiles_x, t1 = t0 + tiles_x;
  bool any = false;
  if (s_start) any = any || s_start[t1] > s_start[t0];
  if (r_start) any = any || r_start[t1] > r_start[t0];
  flags[i] = any ? 1 : 0;
}

// Exclusive scan of count[0..n) into start[0..n] by one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_points_scan(const int *__restrict__ count,
                                                     int *__restrict__ start, int n) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
  int sum = 0;
  for (int k = lo; k < hi; ++k) sum += count[k];
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;
  for (int k = lo; k < hi; ++k) {
    start[k] = run;
    run += count[k];
  }
  if (t == 1023) start[n] = part[1023];
}

// Place each entry at start[tile] + (its rank among earlier entries of the
// same shot and tile), so every tile lists its entries in ascending order.
__global__ void k_points_fill(const int64_t *__restrict__ idx, int n_per_shot, int n_shots,
                              int64_t N, int nx, PointTiles pt, const int *__restrict__ start,
                              int *__restrict__ cell,
                              int *__restrict__ ent) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_per_shot * n_shots) return;
  const int64_t v = idx[e];
  if (v < 0 || v >= N) return;
  const int s = e / n_per_shot;
  const int tile = point_tile_of(v, s, nx, pt);
  int rank = 0;
  for (int e2 = s * n_per_shot; e2 < e; ++e2) {
    const int64_t v2 = idx[e2];
    if (v2 >= 0 && v2 < N && point_tile_of(v2, s, nx, pt) == tile) ++rank;
  }
  const int pos = start[tile] + rank;
  cell[pos] = (int)v;
  ent[pos] = e;
}

}  // namespace tb
