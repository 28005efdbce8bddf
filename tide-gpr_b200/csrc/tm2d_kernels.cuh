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
// for each 32x8 tile of each shot, the list of point entries that fall in it
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

constexpr int kTileX = 32;  // CTA tile of the cell kernels (x fastest)
constexpr int kTileY = 8;

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
// Forward H half-step (maxwell_tm_core.cuh:448-502).  Grid covers the update
// domain [P, n-P+1)^2 with 32x8 tiles; grid.z = shot.
template <typename T, int ST>
__global__ void __launch_bounds__(256)
k_fwd_h(TMGeom<T> g, const T *__restrict__ cq, const T *__restrict__ ey, T *__restrict__ hx,
        T *__restrict__ hz, T *__restrict__ m_ey_x, T *__restrict__ m_ey_z) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x + P;
  const int y = blockIdx.y * kTileY + threadIdx.y + P;
  const int s = blockIdx.z;
  if (x >= g.nx - P + 1 || y >= g.ny - P + 1) return;
  const int64_t j = (int64_t)y * g.nx + x;
  const int64_t i = (int64_t)s * g.N + j;
  const T cqv = g.cq_b ? ldg(cq + i) : ldg(cq + j);
  if (y < g.ny - P) {
    T d = d_yh1<T, ST>(ey, i, g.nx, g.rdy);
    if (y < g.pml_y0 || y >= g.pml_y1h) {
      const T m = ldg(g.byh + y) * m_ey_z[i] + ldg(g.ayh + y) * d;
      m_ey_z[i] = m;
      d = d / ldg(g.kyh + y) + m;
    }
    hx[i] = hx[i] - cqv * d;
  }
  if (x < g.nx - P) {
    T d = d_xh1<T, ST>(ey, i, g.rdx);
    if (x < g.pml_x0 || x >= g.pml_x1h) {
      const T m = ldg(g.bxh + x) * m_ey_x[i] + ldg(g.axh + x) * d;
      m_ey_x[i] = m;
      d = d / ldg(g.kxh + x) + m;
    }
    hz[i] = hz[i] + cqv * d;
  }
}

// Debye (1..n poles) state for the E kernel; n_poles == 0 disables it.
template <typename T> struct DebyeArgs {
  const T *a, *b, *cp;  // [n_poles, ny, nx]
  T *pol;               // [n_shots, n_poles, ny, nx]
  int n_poles;
};

// Forward E half-step with optional snapshot storage, Debye polarisation,
// source injection and receiver recording
// (maxwell_tm_core.cuh:504-599, maxwell_tm_cuda_inst.cu:382-457,
// maxwell.cu:89-141).  Grid covers the full [0,ny)x[0,nx) grid so that points
// outside the update domain are still injected and recorded.
template <typename T, int ST, typename S>
__global__ void __launch_bounds__(256)
k_fwd_e(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cb, const T *__restrict__ hx,
        const T *__restrict__ hz, T *__restrict__ ey, T *__restrict__ m_hx_z,
        T *__restrict__ m_hz_x, S *__restrict__ ey_store, S *__restrict__ curl_store,
        DebyeArgs<T> db, PointCSR src, PointCSR rec, const T *__restrict__ f_t,
        T *__restrict__ r_t) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x;
  const int y = blockIdx.y * kTileY + threadIdx.y;
  const int s = blockIdx.z;
  const int tile = (s * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const bool pts = !point_tile_empty(src, rec, tile);
  if (x >= g.nx || y >= g.ny) return;
  const bool dom = x >= P && y >= P && x < g.nx - P + 1 && y < g.ny - P + 1;
  if (!dom && !pts) return;
  const int64_t j = (int64_t)y * g.nx + x;
  const int64_t i = (int64_t)s * g.N + j;
  const T e_old = ey[i];
  T e_new = e_old;
  if (dom) {
    const T cav = g.ca_b ? ldg(ca + i) : ldg(ca + j);
    const T cbv = g.cb_b ? ldg(cb + i) : ldg(cb + j);
    T dhz_dx = d_x1<T, ST>(hz, i, g.rdx);
    T dhx_dz = d_y1<T, ST>(hx, i, g.nx, g.rdy);
    if (x < g.pml_x0 || x >= g.pml_x1) {
      const T m = ldg(g.bx + x) * m_hz_x[i] + ldg(g.ax + x) * dhz_dx;
      m_hz_x[i] = m;
      dhz_dx = dhz_dx / ldg(g.kx + x) + m;
    }
    if (y < g.pml_y0 || y >= g.pml_y1) {
      const T m = ldg(g.by + y) * m_hx_z[i] + ldg(g.ay + y) * dhx_dz;
      m_hx_z[i] = m;
      dhx_dz = dhx_dz / ldg(g.ky + y) + m;
    }
    const T curl = dhz_dx - dhx_dz;
    if (ey_store) ey_store[i] = Codec<S, T>::enc(e_old);
    if (curl_store) curl_store[i] = Codec<S, T>::enc(curl);
    e_new = cav * e_old + cbv * curl;
    if (db.n_poles > 0) {
      T pol_term = (T)0;
      for (int p = 0; p < db.n_poles; ++p)
        pol_term = pol_term + ldg(db.cp + (int64_t)p * g.N + j) *
                                  db.pol[((int64_t)s * db.n_poles + p) * g.N + j];
      e_new = e_new + pol_term;
    }
  }
  if (pts) e_new = point_accumulate(src, tile, (int)j, f_t, e_new);
  if (dom || pts) ey[i] = e_new;
  if (dom && db.n_poles > 0) {
    const T e_sum = e_new + e_old;
    for (int p = 0; p < db.n_poles; ++p) {
      const int64_t c = (int64_t)p * g.N + j;
      const int64_t pi = ((int64_t)s * db.n_poles + p) * g.N + j;
      db.pol[pi] = ldg(db.a + c) * db.pol[pi] + ldg(db.b + c) * e_sum;
    }
  }
  if (pts) point_record(rec, tile, (int)j, r_t, e_new);
}

// ---------------------------------------------------------------------------
// Exact adjoint, E-phase (maxwell_tm_cuda_inst.cu:954-1027) with the
// coefficient gradient of the previous (later-in-time) step fused in
// (maxwell_tm_cuda_inst.cu:834-871).  lam_ey is not modified here, so at
// iteration t it still holds the final adjoint of step t+1, which is exactly
// what coeff_grad(t+1) consumes.
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

template <typename T, typename S> struct GradArgs {
  const S *ey_st;  // snapshot Ey^t of the step being imaged (nullptr: skip)
  const S *cu_st;  // snapshot curl H^t
  T *acc_ca;       // [n_shots, ny, nx] accumulators
  T *acc_cb;
  T kscale;        // gradient sampling interval as T
};

template <typename T, typename S>
__device__ __forceinline__ void coeff_grad_cell(const GradArgs<T, S> &ga, int64_t i, T lam) {
  if (ga.ey_st) ga.acc_ca[i] = ga.acc_ca[i] + lam * Codec<S, T>::dec(ga.ey_st[i]) * ga.kscale;
  if (ga.cu_st) ga.acc_cb[i] = ga.acc_cb[i] + lam * Codec<S, T>::dec(ga.cu_st[i]) * ga.kscale;
}

template <typename T, int ST, typename S>
__global__ void __launch_bounds__(256)
k_adj_e(TMGeom<T> g, const T *__restrict__ cb, const T *__restrict__ lam_ey,
        T *__restrict__ lam_hx, T *__restrict__ lam_hz, const T *__restrict__ m_hx_z,
        const T *__restrict__ m_hz_x, T *__restrict__ m_hx_z_n, T *__restrict__ m_hz_x_n,
        GradArgs<T, S> ga) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x + P;
  const int y = blockIdx.y * kTileY + threadIdx.y + P;
  const int s = blockIdx.z;
  if (x >= g.nx - P + 1 || y >= g.ny - P + 1) return;
  const int64_t base = (int64_t)s * g.N;
  const int64_t j = (int64_t)y * g.nx + x, i = base + j;
  const T lam = ldg(lam_ey + i);
  coeff_grad_cell(ga, i, lam);
  const T q = (g.cb_b ? ldg(cb + i) : ldg(cb + j)) * lam;
  const bool px = x < g.pml_x0 || x >= g.pml_x1;
  const bool py = y < g.pml_y0 || y >= g.pml_y1;
  m_hz_x_n[i] = px ? ldg(g.bx + x) * ldg(m_hz_x + i) + q : (T)0;
  m_hx_z_n[i] = py ? ldg(g.by + y) * ldg(m_hx_z + i) - q : (T)0;
  T ax_ = (T)FD<ST>::c(0) * (raw_x<T, ST>(g, cb, lam_ey, m_hz_x, base, y, x) -
                            raw_x<T, ST>(g, cb, lam_ey, m_hz_x, base, y, x + 1));
#pragma unroll
  for (int m = 1; m < P; ++m)
    ax_ = ax_ + (T)FD<ST>::c(m) * (raw_x<T, ST>(g, cb, lam_ey, m_hz_x, base, y, x - m) -
                                   raw_x<T, ST>(g, cb, lam_ey, m_hz_x, base, y, x + 1 + m));
  lam_hz[i] = lam_hz[i] + ax_ * g.rdx;
  T ay_ = (T)FD<ST>::c(0) * (raw_y<T, ST>(g, cb, lam_ey, m_hx_z, base, y, x) -
                            raw_y<T, ST>(g, cb, lam_ey, m_hx_z, base, y + 1, x));
#pragma unroll
  for (int m = 1; m < P; ++m)
    ay_ = ay_ + (T)FD<ST>::c(m) * (raw_y<T, ST>(g, cb, lam_ey, m_hx_z, base, y - m, x) -
                                   raw_y<T, ST>(g, cb, lam_ey, m_hx_z, base, y + 1 + m, x));
  lam_hx[i] = lam_hx[i] + ay_ * g.rdy;
}

// Coefficient gradient alone, for the earliest step of a backward call.
template <typename T, int ST, typename S>
__global__ void __launch_bounds__(256)
k_coeff_grad(TMGeom<T> g, const T *__restrict__ lam_ey, GradArgs<T, S> ga) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x + P;
  const int y = blockIdx.y * kTileY + threadIdx.y + P;
  const int s = blockIdx.z;
  if (x >= g.nx - P + 1 || y >= g.ny - P + 1) return;
  const int64_t i = (int64_t)s * g.N + (int64_t)y * g.nx + x;
  coeff_grad_cell(ga, i, ldg(lam_ey + i));
}

// ---------------------------------------------------------------------------
// Exact adjoint, H-phase (maxwell_tm_cuda_inst.cu:1082-1165), with the
// adjoint-source injection at receivers and the source-gradient recording
// (maxwell.cu:107-161) fused as a per-cell epilogue.
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

template <typename T, int ST>
__global__ void __launch_bounds__(256)
k_adj_h(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cq,
        const T *__restrict__ lam_hx, const T *__restrict__ lam_hz, T *__restrict__ lam_ey,
        const T *__restrict__ m_ey_x, const T *__restrict__ m_ey_z, T *__restrict__ m_ey_x_n,
        T *__restrict__ m_ey_z_n, PointCSR rec, PointCSR src, const T *__restrict__ gr_t,
        T *__restrict__ gf_t) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x;
  const int y = blockIdx.y * kTileY + threadIdx.y;
  const int s = blockIdx.z;
  const int tile = (s * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const bool pts = !point_tile_empty(src, rec, tile);
  if (x >= g.nx || y >= g.ny) return;
  const bool dom = x >= P && y >= P && x < g.nx - P + 1 && y < g.ny - P + 1;
  if (!dom && !pts) return;
  const int64_t base = (int64_t)s * g.N;
  const int64_t j = (int64_t)y * g.nx + x, i = base + j;
  T lam = lam_ey[i];
  if (dom) {
    const T cqv = g.cq_b ? ldg(cq + i) : ldg(cq + j);
    const bool py = y < g.pml_y0 || y >= g.pml_y1h;
    const bool px = x < g.pml_x0 || x >= g.pml_x1h;
    const T adj_y = -cqv * ldg(lam_hx + i);
    const T adj_x = cqv * ldg(lam_hz + i);
    m_ey_z_n[i] = (y < g.ny - P && py) ? ldg(g.byh + y) * ldg(m_ey_z + i) + adj_y : (T)0;
    m_ey_x_n[i] = (x < g.nx - P && px) ? ldg(g.bxh + x) * ldg(m_ey_x + i) + adj_x : (T)0;
    const T cav = g.ca_b ? ldg(ca + i) : ldg(ca + j);
    lam = cav * lam;
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
    lam = lam + (dz * g.rdy + dx * g.rdx);
  }
  if (pts) lam = point_accumulate(rec, tile, (int)j, gr_t, lam);
  lam_ey[i] = lam;
  if (pts) point_record(src, tile, (int)j, gf_t, lam);
}

// Shot reduction of the per-shot accumulators (maxwell_tm_inst.cpp:2185-2206):
// grad[j] += sum over shots, summed in shot order.
template <typename T, int ST>
__global__ void __launch_bounds__(256)
k_combine(TMGeom<T> g, T *__restrict__ grad, const T *__restrict__ acc) {
  constexpr int P = FD<ST>::P;
  const int x = blockIdx.x * kTileX + threadIdx.x + P;
  const int y = blockIdx.y * kTileY + threadIdx.y + P;
  if (x >= g.nx - P + 1 || y >= g.ny - P + 1) return;
  const int64_t j = (int64_t)y * g.nx + x;
  T sum = (T)0;
  for (int s = 0; s < g.n_shots; ++s) sum = sum + ldg(acc + (int64_t)s * g.N + j);
  grad[j] = grad[j] + sum;
}

// ---------------------------------------------------------------------------
// Point-list construction (once per call).  Entries with a negative index are
// skipped as in the reference; an index at or beyond ny*nx sets the device
// error word and is skipped instead of writing out of bounds.
__device__ __forceinline__ int point_tile_of(int64_t idx, int s, int nx, int tiles_x,
                                             int tiles_y) {
  const int y = (int)(idx / nx), x = (int)(idx % nx);
  return (s * tiles_y + y / kTileY) * tiles_x + x / kTileX;
}

__global__ void k_points_count(const int64_t *__restrict__ idx, int n_per_shot, int n_shots,
                               int64_t N, int nx, int tiles_x, int tiles_y,
                               int *__restrict__ count) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_per_shot * n_shots) return;
  const int64_t v = idx[e];
  if (v < 0) return;
  if (v >= N) {
    atomicOr(&g_tide_dev_err, 1);
    return;
  }
  atomicAdd(count + point_tile_of(v, e / n_per_shot, nx, tiles_x, tiles_y), 1);
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
                              int64_t N, int nx, int tiles_x, int tiles_y,
                              const int *__restrict__ start, int *__restrict__ cell,
                              int *__restrict__ ent) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_per_shot * n_shots) return;
  const int64_t v = idx[e];
  if (v < 0 || v >= N) return;
  const int s = e / n_per_shot;
  const int tile = point_tile_of(v, s, nx, tiles_x, tiles_y);
  int rank = 0;
  for (int e2 = s * n_per_shot; e2 < e; ++e2) {
    const int64_t v2 = idx[e2];
    if (v2 >= 0 && v2 < N && point_tile_of(v2, s, nx, tiles_x, tiles_y) == tile) ++rank;
  }
  const int pos = start[tile] + rank;
  cell[pos] = (int)v;
  ent[pos] = e;
}

}  // namespace tb
