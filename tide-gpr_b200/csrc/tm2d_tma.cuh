// One-sweep TM2D time steps (stencil order 2, FP32) on TMA-staged tiles.
//
// Each time step is ONE launch that reads every field once and writes it
// once: the two half steps of the forward (H then E), or of the exact
// adjoint (E-phase then H-phase), run back to back on a tile held in shared
// memory.  The E update of a tile needs the new H of one row above and one
// column left of the tile, which belong to neighbouring tiles; they are
// recomputed from the old state (a one-cell halo), so no grid-wide barrier
// is needed between the half steps.  Old and new states therefore live in
// two complete copies (ping-pong) in a pitched internal layout: rows of
// `pitch` floats (a multiple of 32), column x at offset x, shots one after
// another.  The CPML memories that the halo recompute reads are ping-ponged
// too: in the forward the two H-phase memories (a second copy made here), in
// the adjoint all four (the caller's arrays and adjoint_memory_scratch, as
// the reference's backward lays them out).
//
// Data movement.  A tile is TY rows x 64 columns.  Its three fields (with
// the halo) arrive in shared memory by 3-D tiled TMA loads (tensor maps over
// this GPU's pitched buffers; elements outside the grid read as zero), one
// mbarrier per pipeline stage; the model coefficients of a tile arrive the
// same way once per tile.  Results go back with coalesced 8-byte stores;
// snapshots (caller layout, rows of nx cells at any alignment) with
// streaming scalar stores / loads.
//
// Schedule.  The grid is persistent: P CTAs (one per SM; P <= tiles), CTA c
// owns the units [c U / P, (c+1) U / P) of the tile-major sequence of
// U = tiles x shots (tile, shot) units, so every CTA gets the same work to
// within one unit, and a TMA pipeline of kQStages units runs across tile
// boundaries.  A tile's shots are processed in ascending order, so the
// adjoint's coefficient gradient is the kernels' step-major shot sum
// (grad += ((0 + t_0) + t_1) + ...), bit-identical to the other stencil-2
// kernels and to the oracle in that order.  A tile whose shots are split
// between CTA c-1 (shots [0, k), processed first) and CTA c (shots [k, S),
// processed last) hands the running sums over through global memory: CTA
// c-1 stores them and releases a flag, CTA c acquires it (a bounded wait,
// normally long satisfied) and continues the sums.
//
// Numerics.  Every cell value is computed with the same operations in the
// same order as tm2d_s2.cuh (--fmad=false), so fields, snapshots, receivers,
// source gradients and the model gradient are bit-identical to that path.
#pragma once

#include "tb_tma.cuh"
#include "tm2d_kernels.cuh"

namespace tb {

constexpr int kQX = 64;            // tile width (cells)
constexpr int kQThreads = 512;     // 16 warps per CTA
constexpr int kQWarps = kQThreads / 32;
constexpr int kQStages = 3;        // TMA pipeline depth (units in flight)
constexpr uint32_t kQWaitLimit = 1u << 24;  // bounded waits (polls)

// Shared-memory extents (floats) of the staged boxes for a tile of TY rows.
template <int TY> struct QBox {
  static constexpr int EW = kQX + 8, EH = TY + 2;  // rows y0-1..y0+TY,   cols x0-4..x0+67
  static constexpr int XW = kQX, XH = TY + 1;      // rows y0-1..y0+TY-1, cols x0..x0+63
  static constexpr int ZW = kQX + 4, ZH = TY;      // rows y0..y0+TY-1,   cols x0-4..x0+63
  static constexpr int OW = kQX, OH = TY;          // own cells
  static constexpr int QW = kQX + 4, QH = TY + 1;  // rows y0-1..y0+TY-1, cols x0-4..x0+63
  static constexpr int rb(int n) { return (n * 4 + 127) / 128 * 128; }
  static constexpr int E_B = rb(EW * EH), X_B = rb(XW * XH), Z_B = rb(ZW * ZH),
                       O_B = rb(OW * OH), Q_B = rb(QW * QH);
  static constexpr int STAGE_B = E_B + X_B + Z_B;  // one unit's fields
  // coefficient slot: adjoint (ca own, cb E-box, cq Q-box); forward (cq, ca, cb own)
  static constexpr int COEF_ADJ_B = O_B + E_B + Q_B;
  static constexpr int COEF_FWD_B = Q_B + O_B + O_B;
  static constexpr int EXTRA_B = X_B + Z_B + O_B;  // new Hx, new Hz, point pass
  static constexpr int smem_bytes(bool adj) {
    return kQStages * (STAGE_B + (adj ? COEF_ADJ_B : COEF_FWD_B)) + EXTRA_B + 8 * kQStages;
  }
  // transaction bytes of the boxes
  static constexpr uint32_t FIELD_TX = 4u * (EW * EH + XW * XH + ZW * ZH);
  static constexpr uint32_t COEF_ADJ_TX = 4u * (OW * OH + EW * EH + QW * QH);
  static constexpr uint32_t COEF_FWD_TX = 4u * (QW * QH + 2 * OW * OH);
};

// Unit schedule of one CTA: segment A = the first shots [0, nA) of the tile
// its range ends in (processed first; hands its running sums to CTA c+1),
// segment B = whole tiles, segment C = the last shots [cC0, S) of the tile
// its range starts in (processed last; continues CTA c-1's sums).  Requires
// P <= tiles, so that a range spans at least S units and a tile is split
// between at most two CTAs.
struct QSched {
  int S;
  int nA, nB, nC;
  int tA, tB0, tC, cC0;
  __device__ __forceinline__ int n() const { return nA + nB + nC; }
  // (tile, shot, ordinal of the tile in this CTA's sequence, segment 0/1/2)
  __device__ __forceinline__ void unit(int i, int &tile, int &shot, int &ord, int &seg) const {
    const int oA = nA > 0 ? 1 : 0;
    if (i < nA) {
      tile = tA; shot = i; ord = 0; seg = 0;
      return;
    }
    i -= nA;
    if (i < nB) {
      tile = tB0 + i / S; shot = i % S; ord = oA + i / S; seg = 1;
      return;
    }
    i -= nB;
    tile = tC; shot = cC0 + i; ord = oA + nB / S; seg = 2;
  }
};
__device__ __forceinline__ QSched q_sched(int c, int P, int tiles, int S) {
  QSched q;
  const int64_t U = (int64_t)tiles * S;
  const int64_t lo = U * c / P, hi = U * (c + 1) / P;
  q.S = S;
  if (lo % S) {
    q.tC = (int)(lo / S); q.cC0 = (int)(lo % S); q.nC = S - q.cC0;
  } else {
    q.tC = -1; q.cC0 = 0; q.nC = 0;
  }
  if (hi % S) {
    q.tA = (int)(hi / S); q.nA = (int)(hi % S);
  } else {
    q.tA = -1; q.nA = 0;
  }
  const int64_t fa = (lo + S - 1) / S, fb = hi / S;
  q.tB0 = (int)fa;
  q.nB = fb > fa ? (int)((fb - fa) * S) : 0;
  return q;
}

// Shared memory carve-up: kQStages field stages, kQStages coefficient
// slots, the new-H tiles, the point-pass tile and the stage barriers.  Stage
// addresses are computed, not tabulated, so nothing is indexed dynamically
// in local memory.
template <int TY, bool ADJ> struct QSmem {
  using B = QBox<TY>;
  static constexpr int COEF_B = ADJ ? B::COEF_ADJ_B : B::COEF_FWD_B;
  static constexpr int COEF0 = kQStages * B::STAGE_B;
  static constexpr int EXTRA0 = COEF0 + kQStages * COEF_B;
  unsigned char *base;
  float *hxn, *hzn, *ve;
  uint64_t *full;
  __device__ __forceinline__ explicit QSmem(unsigned char *b) : base(b) {
    hxn = reinterpret_cast<float *>(b + EXTRA0);
    hzn = reinterpret_cast<float *>(b + EXTRA0 + B::X_B);
    ve = reinterpret_cast<float *>(b + EXTRA0 + B::X_B + B::Z_B);
    full = reinterpret_cast<uint64_t *>(b + EXTRA0 + B::EXTRA_B);
  }
  __device__ __forceinline__ float *e(int k) const {
    return reinterpret_cast<float *>(base + k * B::STAGE_B);
  }
  __device__ __forceinline__ float *x(int k) const {
    return reinterpret_cast<float *>(base + k * B::STAGE_B + B::E_B);
  }
  __device__ __forceinline__ float *z(int k) const {
    return reinterpret_cast<float *>(base + k * B::STAGE_B + B::E_B + B::X_B);
  }
  // adjoint: c0 = ca (own box), c1 = cb (E box), c2 = cq (Q box);
  // forward: c0 = cq (Q box), c1 = ca (own box), c2 = cb (own box)
  __device__ __forceinline__ float *c0(int k) const {
    return reinterpret_cast<float *>(base + COEF0 + k * COEF_B);
  }
  __device__ __forceinline__ float *c1(int k) const {
    return reinterpret_cast<float *>(base + COEF0 + k * COEF_B + (ADJ ? B::O_B : B::Q_B));
  }
  __device__ __forceinline__ float *c2(int k) const {
    return reinterpret_cast<float *>(base + COEF0 + k * COEF_B +
                                     (ADJ ? B::O_B + B::E_B : B::Q_B + B::O_B));
  }
};

// Tensor maps of one launch (field maps of the current ping-pong copy).
struct QMaps {
  CUtensorMap e, x, z;     // Ey / lEy (E box), Hx / lHx (X box), Hz / lHz (Z box)
  CUtensorMap c0, c1, c2;  // adjoint: ca (own), cb (E box), cq (Q box); forward: cq, ca, cb
};

// Arguments common to both kernels.
struct QCommon {
  TMGeom<float> g;
  int tiles_x, tiles_y, P;
  int64_t pitch, pshot;  // floats per pitched row / per pitched shot
  float *ey_n, *hx_n, *hz_n;  // next copy (pitched)
  PointCSR p0, p1;            // forward: sources, receivers; adjoint: receivers, sources
  const float *v0;            // forward: f_t; adjoint: grad_r_t
  float *v1;                  // forward: r_t; adjoint: grad_f_t
};

struct QFwdArgs {
  QCommon c;
  const float *mex_c, *mez_c;  // H-phase memories, current (caller layout)
  float *mex_n, *mez_n;        // ... next
  float *mhx, *mhz;            // E-phase memories (in place)
  void *ey_st, *cu_st;         // snapshots of this step (caller layout) or null
};

struct QAdjArgs {
  QCommon c;
  const float *mhz_c, *mhx_c, *mex_c, *mez_c;  // l-memories, current
  float *mhz_n, *mhx_n, *mex_n, *mez_n;        // ... next
  const void *ey_st, *cu_st;                   // snapshots of this step or null
  int bg_shots;                                // shots of the snapshot history
  float *grad_ca, *grad_cb;                    // [ny, nx]
  float kscale;
  float *hand;  // [P][2][TY * 64] running sums handed from CTA c-1 to c
  int *flags;   // [P]
  int epoch;    // distinct per launch within a call (flags start at 0)
};

// Issue the TMA loads of unit (tile, shot) into stage k (thread 0 only).
template <int TY, bool ADJ>
__device__ __forceinline__ void q_issue(const QSmem<TY, ADJ> &sm, const QMaps &m, int k, int tile,
                                        int shot, bool coef, int cslot, int tiles_x) {
  using B = QBox<TY>;
  const int y0 = (tile / tiles_x) * TY, x0 = (tile % tiles_x) * kQX;
  uint64_t *bar = sm.full + k;
  fence_proxy_async_smem();
  mbar_arrive_expect_tx(bar, B::FIELD_TX + (coef ? (ADJ ? B::COEF_ADJ_TX : B::COEF_FWD_TX) : 0u));
  tma_load_3d(sm.e(k), &m.e, bar, x0 - 4, y0 - 1, shot);
  tma_load_3d(sm.x(k), &m.x, bar, x0, y0 - 1, shot);
  tma_load_3d(sm.z(k), &m.z, bar, x0 - 4, y0, shot);
  if (coef) {
    if (ADJ) {
      tma_load_3d(sm.c0(cslot), &m.c0, bar, x0, y0, 0);
      tma_load_3d(sm.c1(cslot), &m.c1, bar, x0 - 4, y0 - 1, 0);
      tma_load_3d(sm.c2(cslot), &m.c2, bar, x0 - 4, y0 - 1, 0);
    } else {
      tma_load_3d(sm.c0(cslot), &m.c0, bar, x0 - 4, y0 - 1, 0);
      tma_load_3d(sm.c1(cslot), &m.c1, bar, x0, y0, 0);
      tma_load_3d(sm.c2(cslot), &m.c2, bar, x0, y0, 0);
    }
  }
}

// Does (tile, shot) have point entries in either list?
__device__ __forceinline__ bool q_pts(const PointCSR &a, const PointCSR &b, int id) {
  return !point_tile_empty(a, b, id);
}

// Point passes over the own cells of a tile (values v, RPT rows x 2 columns
// per thread).  The tile's list is staged in shared memory in chunks (cell
// as a tile-local index, and the entry's value or index); every thread then
// scans the chunk for entries at its own cells, so entries at one cell are
// applied in entry order and the lists are read with parallel loads.
constexpr int kQPtChunk = 512;
__device__ __forceinline__ int q_local(int cell, int ybase, int nx, int ty) {
  const int d = cell - ybase;
  if (d < 0) return -1;
  const int oy = d / nx, ox = d - oy * nx;
  return (oy < ty && ox < kQX) ? oy * kQX + ox : -1;
}
// v[c] = v[c] + vals[e] for each entry e at cell c, in entry order.
template <int TY, int RPT>
__device__ __forceinline__ void q_points_add(const PointCSR &pl, const float *vals, int pid,
                                             int ybase, int nx, float (&v)[RPT][2], int *s_cell,
                                             float *s_val) {
  if (pl.start == nullptr || vals == nullptr) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = __ldg(pl.start + pid), e = __ldg(pl.start + pid + 1);
  for (int c0 = b; c0 < e; c0 += kQPtChunk) {
    const int n = min(kQPtChunk, e - c0);
    __syncthreads();
    for (int i = tid; i < n; i += kQThreads) {
      s_cell[i] = q_local(__ldg(pl.cell + c0 + i), ybase, nx, TY);
      s_val[i] = __ldg(vals + __ldg(pl.ent + c0 + i));
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int me = (warp + r * kQWarps) * kQX + 2 * lane + q;
        for (int i = 0; i < n; ++i)
          if (s_cell[i] == me) v[r][q] = v[r][q] + s_val[i];
      }
  }
}
// out[e] = v[c] for each entry e at cell c.
template <int TY, int RPT>
__device__ __forceinline__ void q_points_record(const PointCSR &pl, float *out, int pid,
                                                int ybase, int nx, const float (&v)[RPT][2],
                                                int *s_cell, int *s_ent) {
  if (pl.start == nullptr || out == nullptr) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = __ldg(pl.start + pid), e = __ldg(pl.start + pid + 1);
  for (int c0 = b; c0 < e; c0 += kQPtChunk) {
    const int n = min(kQPtChunk, e - c0);
    __syncthreads();
    for (int i = tid; i < n; i += kQThreads) {
      s_cell[i] = q_local(__ldg(pl.cell + c0 + i), ybase, nx, TY);
      s_ent[i] = __ldg(pl.ent + c0 + i);
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int me = (warp + r * kQWarps) * kQX + 2 * lane + q;
        for (int i = 0; i < n; ++i)
          if (s_cell[i] == me) out[s_ent[i]] = v[r][q];
      }
  }
}

// ============================================================== adjoint
//
// Per unit: phase 1 = adjoint E-phase (cb lEy -> lHx, lHz and the x / y
// memories of the E-phase) on the own cells plus the halo row y0-1 (lHx) and
// column x0-1 (lHz), into shared memory; phase 2 = adjoint H-phase (lEy from
// the new lHx / lHz, the H-phase memories), receivers injected, sources
// recorded, image terms summed over the tile's shots.  Formulas: tm2d_s2.cuh
// adj_e_tile / adj_h_tile.
// CPML memory values one cell reads (prefetched before its arithmetic, so a
// strip tile waits for memory once per phase, not once per cell).
struct QM4 {
  float a, b, c, d;
};

template <int TY>
struct QAdjCell {
  using B = QBox<TY>;
  // Strip tests of the E-phase (integer grid) and H-phase (half grid).
  static __device__ __forceinline__ bool xs(const TMGeom<float> &g, int x) {
    return !(x >= g.pml_x0 && x < g.pml_x1);
  }
  static __device__ __forceinline__ bool ys(const TMGeom<float> &g, int y) {
    return !(y >= g.pml_y0 && y < g.pml_y1);
  }
  static __device__ __forceinline__ bool xsh(const TMGeom<float> &g, int x) {
    return !(x >= g.pml_x0 && x < g.pml_x1h);
  }
  static __device__ __forceinline__ bool ysh(const TMGeom<float> &g, int y) {
    return !(y >= g.pml_y0 && y < g.pml_y1h);
  }
  // phase-1 memories of cell (y, x): l-hz_x at x and x + 1, l-hx_z at y and y + 1
  static __device__ __forceinline__ QM4 e_loads(const QAdjArgs &a, int y, int x, int64_t sb) {
    const TMGeom<float> &g = a.c.g;
    QM4 m{0.f, 0.f, 0.f, 0.f};
    if (y < 1 || x < 1 || y >= g.ny || x >= g.nx) return m;
    const int64_t j = sb + (int64_t)y * g.nx + x;
    if (xs(g, x)) m.a = a.mhz_c[j];
    if (x + 1 < g.nx && xs(g, x + 1)) m.b = a.mhz_c[j + 1];
    if (ys(g, y)) m.c = a.mhx_c[j];
    if (y + 1 < g.ny && ys(g, y + 1)) m.d = a.mhx_c[j + g.nx];
    return m;
  }
  // phase 1 at cell (y, x): new lHx and lHz; own cells also write the next
  // E-phase memories.
  template <bool IN>
  static __device__ __forceinline__ void e_phase(const QAdjArgs &a, const float *E,
                                                 const float *CB, float lhx, float lhz, int y,
                                                 int x, int y0, int x0, int64_t sb, bool own,
                                                 const QM4 &m, float &hx_new, float &hz_new) {
    const TMGeom<float> &g = a.c.g;
    const int ly = y - y0 + 1, lx = x - x0 + 4;  // E-box coordinates
    const float q = CB[ly * B::EW + lx] * E[ly * B::EW + lx];
    const float qr = CB[ly * B::EW + lx + 1] * E[ly * B::EW + lx + 1];
    const float q1 = CB[(ly + 1) * B::EW + lx] * E[(ly + 1) * B::EW + lx];
    if (IN) {
      hz_new = lhz + ((float)1 * (q - qr)) * g.rdx;
      hx_new = lhx + ((float)1 * ((-q) - (-q1))) * g.rdy;
      return;
    }
    hx_new = lhx;
    hz_new = lhz;
    if (y < 1 || x < 1 || y >= g.ny || x >= g.nx) return;
    const int64_t j = sb + (int64_t)y * g.nx + x;
    float rx, rxr, ry0, ry1;
    if (!xs(g, x)) {
      rx = q;
    } else {
      const float mn = __ldg(g.bx + x) * m.a + q;
      rx = __ldg(g.ax + x) * mn + q / __ldg(g.kx + x);
      if (own) a.mhz_n[j] = mn;
    }
    if (x + 1 >= g.nx) {
      rxr = 0.f;
    } else if (!xs(g, x + 1)) {
      rxr = qr;
    } else {
      const float mn = __ldg(g.bx + x + 1) * m.b + qr;
      rxr = __ldg(g.ax + x + 1) * mn + qr / __ldg(g.kx + x + 1);
    }
    if (!ys(g, y)) {
      ry0 = -q;
    } else {
      const float mn = __ldg(g.by + y) * m.c - q;
      ry0 = __ldg(g.ay + y) * mn - q / __ldg(g.ky + y);
      if (own) a.mhx_n[j] = mn;
    }
    if (y + 1 >= g.ny) {
      ry1 = 0.f;
    } else if (!ys(g, y + 1)) {
      ry1 = -q1;
    } else {
      const float mn = __ldg(g.by + y + 1) * m.d - q1;
      ry1 = __ldg(g.ay + y + 1) * mn - q1 / __ldg(g.ky + y + 1);
    }
    hz_new = lhz + ((float)1 * (rx - rxr)) * g.rdx;
    hx_new = lhx + ((float)1 * (ry0 - ry1)) * g.rdy;
  }

  // phase-2 memories of cell (y, x): l-ey_z at y - 1 and y, l-ey_x at x and x - 1
  static __device__ __forceinline__ QM4 h_loads(const QAdjArgs &a, int y, int x, int64_t sb) {
    const TMGeom<float> &g = a.c.g;
    QM4 m{0.f, 0.f, 0.f, 0.f};
    if (x < 1 || y < 1 || y >= g.ny || x >= g.nx) return m;
    const int64_t j = sb + (int64_t)y * g.nx + x;
    if (y - 1 >= 1 && y - 1 < g.ny - 1 && ysh(g, y - 1)) m.a = a.mez_c[j - g.nx];
    if (y < g.ny - 1 && ysh(g, y)) m.b = a.mez_c[j];
    if (x < g.nx - 1 && xsh(g, x)) m.c = a.mex_c[j];
    if (x - 1 >= 1 && x - 1 < g.nx - 1 && xsh(g, x - 1)) m.d = a.mex_c[j - 1];
    return m;
  }
  // phase 2 at own cell (y, x): the new lEy before points.
  template <bool IN>
  static __device__ __forceinline__ float h_phase(const QAdjArgs &a, const float *E,
                                                  const float *CA, const float *CQ,
                                                  const float *HXN, const float *HZN, int y, int x,
                                                  int y0, int x0, int64_t sb, const QM4 &m) {
    const TMGeom<float> &g = a.c.g;
    const int oy = y - y0, ox = x - x0;
    const float lam = E[(oy + 1) * B::EW + ox + 4];
    const float ca = CA[oy * B::OW + ox];
    const float cz0 = CQ[oy * B::QW + ox + 4], cz1 = CQ[(oy + 1) * B::QW + ox + 4];
    const float cx = CQ[(oy + 1) * B::QW + ox + 4], cl = CQ[(oy + 1) * B::QW + ox + 3];
    const float h0 = HXN[oy * B::XW + ox], h1 = HXN[(oy + 1) * B::XW + ox];
    const float zx = HZN[oy * B::ZW + ox + 4], zl = HZN[oy * B::ZW + ox + 3];
    if (IN) {
      const float rz0 = -cz0 * h0, rz1 = -cz1 * h1;
      const float rx = cx * zx, rxl = cl * zl;
      float v = ca * lam;
      v = v + (((float)1 * (rz0 - rz1)) * g.rdy + ((float)1 * (rxl - rx)) * g.rdx);
      return v;
    }
    if (x < 1 || y < 1 || y >= g.ny || x >= g.nx) return lam;
    const int64_t j = sb + (int64_t)y * g.nx + x;
    float rz0 = 0.f, rz1 = 0.f, rx = 0.f, rxl = 0.f;
    {  // row y - 1
      const int yy = y - 1;
      if (yy >= 1 && yy < g.ny - 1) {
        const float adj = -cz0 * h0;
        if (!ysh(g, yy)) {
          rz0 = adj;
        } else {
          const float mn = __ldg(g.byh + yy) * m.a + adj;
          rz0 = __ldg(g.ayh + yy) * mn + adj / __ldg(g.kyh + yy);
        }
      }
    }
    if (y < g.ny - 1) {  // row y (y >= 1 here)
      const float adj = -cz1 * h1;
      if (!ysh(g, y)) {
        rz1 = adj;
      } else {
        const float mn = __ldg(g.byh + y) * m.b + adj;
        rz1 = __ldg(g.ayh + y) * mn + adj / __ldg(g.kyh + y);
        a.mez_n[j] = mn;
      }
    }
    if (x < g.nx - 1) {  // column x (x >= 1 here)
      const float adj = cx * zx;
      if (!xsh(g, x)) {
        rx = adj;
      } else {
        const float mn = __ldg(g.bxh + x) * m.c + adj;
        rx = __ldg(g.axh + x) * mn + adj / __ldg(g.kxh + x);
        a.mex_n[j] = mn;
      }
    }
    {  // column x - 1
      const int xl = x - 1;
      if (xl >= 1 && xl < g.nx - 1) {
        const float adj = cl * zl;
        if (!xsh(g, xl)) {
          rxl = adj;
        } else {
          const float mn = __ldg(g.bxh + xl) * m.d + adj;
          rxl = __ldg(g.axh + xl) * mn + adj / __ldg(g.kxh + xl);
        }
      }
    }
    float v = ca * lam;
    v = v + (((float)1 * (rz0 - rz1)) * g.rdy + ((float)1 * (rxl - rx)) * g.rdx);
    return v;
  }
};

template <typename SN> __device__ __forceinline__ float q_dec(SN v) { return Codec<SN, float>::dec(v); }

// Snapshots of the own cells of unit (tile, shot): shot s images against
// snapshot shot s % bg_shots; cells outside the update domain read nothing.
template <int TY, int RPT, typename SN>
__device__ __forceinline__ void q_snap_load(const QAdjArgs &a, int tile, int shot,
                                            SN (&ev)[RPT][2], SN (&cv)[RPT][2]) {
  const TMGeom<float> &g = a.c.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int y0 = (tile / a.c.tiles_x) * TY, x0 = (tile % a.c.tiles_x) * kQX;
  const int64_t snb = (int64_t)(shot % a.bg_shots) * g.N;
#pragma unroll
  for (int r = 0; r < RPT; ++r)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int y = y0 + warp + r * kQWarps, x = x0 + 2 * lane + q;
      const bool ok = y >= 1 && x >= 1 && y < g.ny && x < g.nx;
      const int64_t j = snb + (int64_t)y * g.nx + x;
      ev[r][q] = (ok && a.ey_st) ? load_stream(static_cast<const SN *>(a.ey_st) + j) : SN(0.f);
      cv[r][q] = (ok && a.cu_st) ? load_stream(static_cast<const SN *>(a.cu_st) + j) : SN(0.f);
    }
}

template <int TY, typename SN>
__global__ void __launch_bounds__(kQThreads, 1)
kq_adj_step(const __grid_constant__ QMaps m, const QAdjArgs a) {
  using B = QBox<TY>;
  using C = QAdjCell<TY>;
  constexpr int RPT = TY / kQWarps;  // own rows per thread (x 2 columns)
  extern __shared__ __align__(128) unsigned char q_smem[];
  const QSmem<TY, true> sm(q_smem);
  const QCommon &cm = a.c;
  const TMGeom<float> &g = cm.g;
  const int S = g.n_shots, nx = g.nx, ny = g.ny;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cta = blockIdx.x;
  const QSched sc = q_sched(cta, cm.P, cm.tiles_x * cm.tiles_y, S);
  const int n_units = sc.n();
  const bool imaging = a.ey_st != nullptr || a.cu_st != nullptr;

  if (tid == 0) {
    for (int k = 0; k < kQStages; ++k) mbar_init(sm.full + k, 1);
    mbar_init_fence();
  }
  __syncthreads();
  // prologue: the first kQStages units
  if (tid == 0) {
    int prev_ord = -1;
    for (int i = 0; i < n_units && i < kQStages; ++i) {
      int tile, shot, ord, seg;
      sc.unit(i, tile, shot, ord, seg);
      q_issue<TY, true>(sm, m, i, tile, shot, ord != prev_ord, ord % kQStages, cm.tiles_x);
      prev_ord = ord;
    }
  }
  float sum_a[RPT][2], sum_b[RPT][2];
  // snapshots are loaded one unit ahead (their latency overlaps a whole unit)
  SN ev[RPT][2], cv[RPT][2];
  if (imaging && n_units > 0) {
    int t0, s0, o0, g0;
    sc.unit(0, t0, s0, o0, g0);
    q_snap_load<TY, RPT, SN>(a, t0, s0, ev, cv);
  }
  int prev_ord = -1;
  for (int i = 0; i < n_units; ++i) {
    int tile, shot, ord, seg;
    sc.unit(i, tile, shot, ord, seg);
    const int k = i % kQStages;
    const int cs = ord % kQStages;
    const int y0 = (tile / cm.tiles_x) * TY, x0 = (tile % cm.tiles_x) * kQX;
    const int64_t sb = (int64_t)shot * g.N;  // shot base, caller layout
    const int64_t pb = (int64_t)shot * cm.pshot;
    const bool first_of_tile = ord != prev_ord;
    prev_ord = ord;
    if (first_of_tile) {
      if (seg == 2 && imaging) {
        // continue the running sums of CTA cta-1 (it processed shots [0, cC0))
        if (tid == 0) {
          const int *f = a.flags + (cta - 1);
          uint32_t it = 0;
          while (ld_acquire_gpu(f) != a.epoch) {
            if (++it > kQWaitLimit) {
              atomicOr(&g_tide_dev_err, 4);
              break;
            }
            __nanosleep(64);
          }
        }
        __syncthreads();
        const float *h = a.hand + (size_t)(cta - 1) * 2 * TY * kQX;
#pragma unroll
        for (int r = 0; r < RPT; ++r)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int o = (warp + r * kQWarps) * kQX + 2 * lane + q;
            sum_a[r][q] = __ldcg(h + o);
            sum_b[r][q] = __ldcg(h + TY * kQX + o);
          }
      } else {
#pragma unroll
        for (int r = 0; r < RPT; ++r) sum_a[r][0] = sum_a[r][1] = sum_b[r][0] = sum_b[r][1] = 0.f;
      }
    }
    SN evn[RPT][2], cvn[RPT][2];
    if (imaging && i + 1 < n_units) {
      int t1, s1, o1, g1;
      sc.unit(i + 1, t1, s1, o1, g1);
      q_snap_load<TY, RPT, SN>(a, t1, s1, evn, cvn);
    }
    // A transfer that never lands ends the wait with the error word set; the
    // CTA still runs every barrier so the launch finishes.
    if (!mbar_wait(sm.full + k, (uint32_t)((i / kQStages) & 1), kQWaitLimit))
      atomicOr(&g_tide_dev_err, 8);
    const float *E = sm.e(k), *LX = sm.x(k), *LZ = sm.z(k);
    const float *CA = sm.c0(cs), *CB = sm.c1(cs), *CQ = sm.c2(cs);
    const bool in = y0 - 1 >= max(1, g.pml_y0) && y0 + TY < min(ny, g.pml_y1) &&
                    x0 - 1 >= max(1, g.pml_x0) && x0 + kQX < min(nx, g.pml_x1);
    // ---------------- phase 1: adjoint E-phase
    // (strip tiles: every memory value the thread's cells read is loaded first)
    QM4 mm[RPT][2], mh[2];
    const QM4 z4{0.f, 0.f, 0.f, 0.f};
    if (!in) {
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::e_loads(a, y0 + warp + r * kQWarps, x0 + 2 * lane + q, sb);
      if (warp == 0) {
        mh[0] = C::e_loads(a, y0 - 1, x0 + 2 * lane, sb);
        mh[1] = C::e_loads(a, y0 - 1, x0 + 2 * lane + 1, sb);
      } else if (warp == 1 && lane < TY) {
        mh[0] = C::e_loads(a, y0 + lane, x0 - 1, sb);
      }
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int oy = warp + r * kQWarps, y = y0 + oy;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = 2 * lane + q, x = x0 + ox;
        const float lhx = LX[(oy + 1) * B::XW + ox], lhz = LZ[oy * B::ZW + ox + 4];
        float hxn, hzn;
        if (in)
          C::template e_phase<true>(a, E, CB, lhx, lhz, y, x, y0, x0, sb, true, z4, hxn, hzn);
        else
          C::template e_phase<false>(a, E, CB, lhx, lhz, y, x, y0, x0, sb, true, mm[r][q], hxn,
                                     hzn);
        sm.hxn[(oy + 1) * B::XW + ox] = hxn;
        sm.hzn[oy * B::ZW + ox + 4] = hzn;
        if (y < ny && x < nx) {
          const int64_t p = pb + (int64_t)y * cm.pitch + x;
          cm.hx_n[p] = hxn;
          cm.hz_n[p] = hzn;
        }
      }
    }
    if (warp == 0) {  // halo row y0 - 1 (new lHx only)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = 2 * lane + q, y = y0 - 1, x = x0 + ox;
        const float lhx = LX[ox];
        float hxn, hzn;
        if (in)
          C::template e_phase<true>(a, E, CB, lhx, 0.f, y, x, y0, x0, sb, false, z4, hxn, hzn);
        else
          C::template e_phase<false>(a, E, CB, lhx, 0.f, y, x, y0, x0, sb, false, mh[q], hxn,
                                     hzn);
        sm.hxn[ox] = hxn;
      }
    } else if (warp == 1 && lane < TY) {  // halo column x0 - 1 (new lHz only)
      const int oy = lane, y = y0 + oy, x = x0 - 1;
      const float lhz = LZ[oy * B::ZW + 3];
      float hxn, hzn;
      if (in)
        C::template e_phase<true>(a, E, CB, 0.f, lhz, y, x, y0, x0, sb, false, z4, hxn, hzn);
      else
        C::template e_phase<false>(a, E, CB, 0.f, lhz, y, x, y0, x0, sb, false, mh[0], hxn, hzn);
      sm.hzn[oy * B::ZW + 3] = hzn;
    }
    __syncthreads();
    // ---------------- phase 2: adjoint H-phase
    const int pid = (shot * cm.tiles_y + tile / cm.tiles_x) * cm.tiles_x + tile % cm.tiles_x;
    const bool pts = q_pts(cm.p0, cm.p1, pid);
    float v[RPT][2];
    if (in) {
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          v[r][q] = C::template h_phase<true>(a, E, CA, CQ, sm.hxn, sm.hzn, y0 + warp + r * kQWarps,
                                              x0 + 2 * lane + q, y0, x0, sb, z4);
    } else {
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::h_loads(a, y0 + warp + r * kQWarps, x0 + 2 * lane + q, sb);
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          v[r][q] = C::template h_phase<false>(a, E, CA, CQ, sm.hxn, sm.hzn,
                                               y0 + warp + r * kQWarps, x0 + 2 * lane + q, y0,
                                               x0, sb, mm[r][q]);
    }
    if (pts) {
      // receivers (lEy += grad_r, entry order), then sources (grad_f = lEy)
      int *s_cell = reinterpret_cast<int *>(sm.ve);
      float *s_val = sm.ve + kQPtChunk;
      const int ybase = y0 * nx + x0;
      q_points_add<TY, RPT>(cm.p0, cm.v0, pid, ybase, nx, v, s_cell, s_val);
      q_points_record<TY, RPT>(cm.p1, cm.v1, pid, ybase, nx, v, s_cell,
                               reinterpret_cast<int *>(s_val));
    }
    // store lEy, image terms
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int y = y0 + warp + r * kQWarps;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int x = x0 + 2 * lane + q;
        if (y < ny && x < nx) {
          cm.ey_n[pb + (int64_t)y * cm.pitch + x] = v[r][q];
          if (imaging && y >= 1 && x >= 1) {
            if (a.ey_st) sum_a[r][q] = sum_a[r][q] + v[r][q] * q_dec(ev[r][q]) * a.kscale;
            if (a.cu_st) sum_b[r][q] = sum_b[r][q] + v[r][q] * q_dec(cv[r][q]) * a.kscale;
          }
        }
      }
    }
    // end of this CTA's part of the tile: hand the sums over or update the gradient
    const bool last_of_tile = (seg == 0) ? (shot == sc.nA - 1) : (shot == S - 1);
    if (imaging && last_of_tile) {
      if (seg == 0) {
        float *h = a.hand + (size_t)cta * 2 * TY * kQX;
#pragma unroll
        for (int r = 0; r < RPT; ++r)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int o = (warp + r * kQWarps) * kQX + 2 * lane + q;
            __stcg(h + o, sum_a[r][q]);
            __stcg(h + TY * kQX + o, sum_b[r][q]);
          }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release_gpu(a.flags + cta, a.epoch);
      } else {
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
          const int y = y0 + warp + r * kQWarps;
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int x = x0 + 2 * lane + q;
            if (y >= 1 && x >= 1 && y < ny && x < nx) {
              const int64_t j = (int64_t)y * nx + x;
              if (a.ey_st) a.grad_ca[j] = a.grad_ca[j] + sum_a[r][q];
              if (a.cu_st) a.grad_cb[j] = a.grad_cb[j] + sum_b[r][q];
            }
          }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        ev[r][q] = evn[r][q];
        cv[r][q] = cvn[r][q];
      }
    __syncthreads();  // stage k and the new-H tiles are free
    if (tid == 0 && i + kQStages < n_units) {
      int t2, s2, o2, g2;
      sc.unit(i + kQStages, t2, s2, o2, g2);
      int op;
      {
        int t1, s1, g1;
        sc.unit(i + kQStages - 1, t1, s1, op, g1);
      }
      q_issue<TY, true>(sm, m, k, t2, s2, o2 != op, o2 % kQStages, cm.tiles_x);
    }
  }
}

// ============================================================== forward
//
// Per unit: phase 1 = H half step (new Hx on rows y0-1..y0+TY-1, new Hz on
// columns x0-1..x0+63; own cells write the next H-phase memories), phase 2 =
// E half step on the own cells (E-phase memories in place), snapshots of
// Ey^n and curl H, sources added, receivers recorded.  Formulas:
// tm2d_s2.cuh fwd_h_tile / fwd_e_tile.
template <int TY>
struct QFwdCell {
  using B = QBox<TY>;
  // H-phase memories of cell (y, x): m_ey_z (a) and m_ey_x (b) where the cell
  // is in their strips
  static __device__ __forceinline__ QM4 h_loads(const QFwdArgs &a, int y, int x, int64_t sb) {
    const TMGeom<float> &g = a.c.g;
    QM4 m{0.f, 0.f, 0.f, 0.f};
    if (y < 1 || x < 1 || y >= g.ny || x >= g.nx) return m;
    const int64_t j = sb + (int64_t)y * g.nx + x;
    if (y < g.ny - 1 && (y < g.pml_y0 || y >= g.pml_y1h)) m.a = a.mez_c[j];
    if (x < g.nx - 1 && (x < g.pml_x0 || x >= g.pml_x1h)) m.b = a.mex_c[j];
    return m;
  }
  // E-phase memories of an own cell: m_hz_x (a) and m_hx_z (b) in their strips
  static __device__ __forceinline__ QM4 e_loads(const QFwdArgs &a, int y, int x, int64_t sb) {
    const TMGeom<float> &g = a.c.g;
    QM4 m{0.f, 0.f, 0.f, 0.f};
    if (y < 1 || x < 1 || y >= g.ny || x >= g.nx) return m;
    const int64_t j = sb + (int64_t)y * g.nx + x;
    if (x < g.pml_x0 || x >= g.pml_x1) m.a = a.mhz[j];
    if (y < g.pml_y0 || y >= g.pml_y1) m.b = a.mhx[j];
    return m;
  }
  template <bool IN>
  static __device__ __forceinline__ void h_phase(const QFwdArgs &a, const float *E,
                                                 const float *CQ, float hx, float hz, int y,
                                                 int x, int y0, int x0, int64_t sb, bool own,
                                                 const QM4 &m, float &hx_new, float &hz_new) {
    const TMGeom<float> &g = a.c.g;
    const int ly = y - y0 + 1, lx = x - x0 + 4;
    const float e0 = E[ly * B::EW + lx], e1 = E[(ly + 1) * B::EW + lx], er = E[ly * B::EW + lx + 1];
    const float c = CQ[ly * B::QW + lx];
    if (IN) {
      hx_new = hx - c * ((e1 - e0) * g.rdy);
      hz_new = hz + c * ((er - e0) * g.rdx);
      return;
    }
    hx_new = hx;
    hz_new = hz;
    if (y < 1 || x < 1 || y >= g.ny || x >= g.nx) return;
    const int64_t j = sb + (int64_t)y * g.nx + x;
    if (y < g.ny - 1) {
      float d = (e1 - e0) * g.rdy;
      if (y < g.pml_y0 || y >= g.pml_y1h) {
        const float mm = __ldg(g.byh + y) * m.a + __ldg(g.ayh + y) * d;
        if (own) a.mez_n[j] = mm;
        d = d / __ldg(g.kyh + y) + mm;
      }
      hx_new = hx - c * d;
    }
    if (x < g.nx - 1) {
      float d = (er - e0) * g.rdx;
      if (x < g.pml_x0 || x >= g.pml_x1h) {
        const float mm = __ldg(g.bxh + x) * m.b + __ldg(g.axh + x) * d;
        if (own) a.mex_n[j] = mm;
        d = d / __ldg(g.kxh + x) + mm;
      }
      hz_new = hz + c * d;
    }
  }
};

template <int TY, typename SN>
__global__ void __launch_bounds__(kQThreads, 1)
kq_fwd_step(const __grid_constant__ QMaps m, const QFwdArgs a) {
  using B = QBox<TY>;
  using C = QFwdCell<TY>;
  constexpr int RPT = TY / kQWarps;
  extern __shared__ __align__(128) unsigned char q_smem[];
  const QSmem<TY, false> sm(q_smem);
  const QCommon &cm = a.c;
  const TMGeom<float> &g = cm.g;
  const int S = g.n_shots, nx = g.nx, ny = g.ny;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const QSched sc = q_sched(blockIdx.x, cm.P, cm.tiles_x * cm.tiles_y, S);
  const int n_units = sc.n();

  if (tid == 0) {
    for (int k = 0; k < kQStages; ++k) mbar_init(sm.full + k, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0) {
    int prev_ord = -1;
    for (int i = 0; i < n_units && i < kQStages; ++i) {
      int tile, shot, ord, seg;
      sc.unit(i, tile, shot, ord, seg);
      q_issue<TY, false>(sm, m, i, tile, shot, ord != prev_ord, ord % kQStages, cm.tiles_x);
      prev_ord = ord;
    }
  }
  for (int i = 0; i < n_units; ++i) {
    int tile, shot, ord, seg;
    sc.unit(i, tile, shot, ord, seg);
    const int k = i % kQStages;
    const int cs = ord % kQStages;
    const int y0 = (tile / cm.tiles_x) * TY, x0 = (tile % cm.tiles_x) * kQX;
    const int64_t sb = (int64_t)shot * g.N;
    const int64_t pb = (int64_t)shot * cm.pshot;
    // A transfer that never lands ends the wait with the error word set; the
    // CTA still runs every barrier so the launch finishes.
    if (!mbar_wait(sm.full + k, (uint32_t)((i / kQStages) & 1), kQWaitLimit))
      atomicOr(&g_tide_dev_err, 8);
    const float *E = sm.e(k), *HX = sm.x(k), *HZ = sm.z(k);
    const float *CQ = sm.c0(cs), *CA = sm.c1(cs), *CB = sm.c2(cs);
    const bool in = y0 - 1 >= max(1, g.pml_y0) && y0 + TY < min(ny, g.pml_y1) &&
                    x0 - 1 >= max(1, g.pml_x0) && x0 + kQX < min(nx, g.pml_x1);
    // ---------------- phase 1: H half step
    // (strip tiles: the memories of the thread's cells are loaded first)
    QM4 mm[RPT][2], mh[2];
    const QM4 z4{0.f, 0.f, 0.f, 0.f};
    if (!in) {
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::h_loads(a, y0 + warp + r * kQWarps, x0 + 2 * lane + q, sb);
      if (warp == 0) {
        mh[0] = C::h_loads(a, y0 - 1, x0 + 2 * lane, sb);
        mh[1] = C::h_loads(a, y0 - 1, x0 + 2 * lane + 1, sb);
      } else if (warp == 1 && lane < TY) {
        mh[0] = C::h_loads(a, y0 + lane, x0 - 1, sb);
      }
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int oy = warp + r * kQWarps, y = y0 + oy;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = 2 * lane + q, x = x0 + ox;
        const float hx = HX[(oy + 1) * B::XW + ox], hz = HZ[oy * B::ZW + ox + 4];
        float hxn, hzn;
        if (in)
          C::template h_phase<true>(a, E, CQ, hx, hz, y, x, y0, x0, sb, true, z4, hxn, hzn);
        else
          C::template h_phase<false>(a, E, CQ, hx, hz, y, x, y0, x0, sb, true, mm[r][q], hxn,
                                     hzn);
        sm.hxn[(oy + 1) * B::XW + ox] = hxn;
        sm.hzn[oy * B::ZW + ox + 4] = hzn;
        if (y < ny && x < nx) {
          const int64_t p = pb + (int64_t)y * cm.pitch + x;
          cm.hx_n[p] = hxn;
          cm.hz_n[p] = hzn;
        }
      }
    }
    if (warp == 0) {  // halo row y0 - 1 (new Hx only)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = 2 * lane + q;
        float hxn, hzn;
        if (in)
          C::template h_phase<true>(a, E, CQ, HX[ox], 0.f, y0 - 1, x0 + ox, y0, x0, sb, false,
                                    z4, hxn, hzn);
        else
          C::template h_phase<false>(a, E, CQ, HX[ox], 0.f, y0 - 1, x0 + ox, y0, x0, sb, false,
                                     mh[q], hxn, hzn);
        sm.hxn[ox] = hxn;
      }
    } else if (warp == 1 && lane < TY) {  // halo column x0 - 1 (new Hz only)
      const int oy = lane;
      float hxn, hzn;
      if (in)
        C::template h_phase<true>(a, E, CQ, 0.f, HZ[oy * B::ZW + 3], y0 + oy, x0 - 1, y0, x0, sb,
                                  false, z4, hxn, hzn);
      else
        C::template h_phase<false>(a, E, CQ, 0.f, HZ[oy * B::ZW + 3], y0 + oy, x0 - 1, y0, x0,
                                   sb, false, mh[0], hxn, hzn);
      sm.hzn[oy * B::ZW + 3] = hzn;
    }
    __syncthreads();
    // ---------------- phase 2: E half step
    const int pid = (shot * cm.tiles_y + tile / cm.tiles_x) * cm.tiles_x + tile % cm.tiles_x;
    const bool pts = q_pts(cm.p0, cm.p1, pid);
    float v[RPT][2];
    if (!in) {
#pragma unroll
      for (int r = 0; r < RPT; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::e_loads(a, y0 + warp + r * kQWarps, x0 + 2 * lane + q, sb);
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int oy = warp + r * kQWarps, y = y0 + oy;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = 2 * lane + q, x = x0 + ox;
        const float eo = E[(oy + 1) * B::EW + ox + 4];
        const float vz = sm.hzn[oy * B::ZW + ox + 4], vzl = sm.hzn[oy * B::ZW + ox + 3];
        const float vx1 = sm.hxn[(oy + 1) * B::XW + ox], vx0 = sm.hxn[oy * B::XW + ox];
        const float ca = CA[oy * B::OW + ox], cb = CB[oy * B::OW + ox];
        float e = eo;
        const bool inside = y < ny && x < nx;
        if (in) {
          const float curl = (vz - vzl) * g.rdx - (vx1 - vx0) * g.rdy;
          const int64_t j = sb + (int64_t)y * nx + x;
          if (a.ey_st) store_stream(static_cast<SN *>(a.ey_st) + j, Codec<SN, float>::enc(eo));
          if (a.cu_st) store_stream(static_cast<SN *>(a.cu_st) + j, Codec<SN, float>::enc(curl));
          e = ca * eo + cb * curl;
        } else if (inside && y >= 1 && x >= 1) {
          const int64_t j = sb + (int64_t)y * nx + x;
          float dz = (vz - vzl) * g.rdx;
          float dy = (vx1 - vx0) * g.rdy;
          if (x < g.pml_x0 || x >= g.pml_x1) {
            const float m1 = __ldg(g.bx + x) * mm[r][q].a + __ldg(g.ax + x) * dz;
            a.mhz[j] = m1;
            dz = dz / __ldg(g.kx + x) + m1;
          }
          if (y < g.pml_y0 || y >= g.pml_y1) {
            const float m1 = __ldg(g.by + y) * mm[r][q].b + __ldg(g.ay + y) * dy;
            a.mhx[j] = m1;
            dy = dy / __ldg(g.ky + y) + m1;
          }
          const float curl = dz - dy;
          if (a.ey_st) store_stream(static_cast<SN *>(a.ey_st) + j, Codec<SN, float>::enc(eo));
          if (a.cu_st) store_stream(static_cast<SN *>(a.cu_st) + j, Codec<SN, float>::enc(curl));
          e = ca * eo + cb * curl;
        }
        v[r][q] = e;
      }
    }
    if (pts) {
      // sources (Ey += f, entry order), then receivers (r = Ey)
      int *s_cell = reinterpret_cast<int *>(sm.ve);
      float *s_val = sm.ve + kQPtChunk;
      const int ybase = y0 * nx + x0;
      q_points_add<TY, RPT>(cm.p0, cm.v0, pid, ybase, nx, v, s_cell, s_val);
      q_points_record<TY, RPT>(cm.p1, cm.v1, pid, ybase, nx, v, s_cell,
                               reinterpret_cast<int *>(s_val));
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int y = y0 + warp + r * kQWarps;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int x = x0 + 2 * lane + q;
        if (y < ny && x < nx) cm.ey_n[pb + (int64_t)y * cm.pitch + x] = v[r][q];
      }
    }
    __syncthreads();  // stage k and the new-H tiles are free
    if (tid == 0 && i + kQStages < n_units) {
      int t2, s2, o2, g2, t1, s1, o1, g1;
      sc.unit(i + kQStages, t2, s2, o2, g2);
      sc.unit(i + kQStages - 1, t1, s1, o1, g1);
      q_issue<TY, false>(sm, m, k, t2, s2, o2 != o1, o2 % kQStages, cm.tiles_x);
    }
  }
}

}  // namespace tb
