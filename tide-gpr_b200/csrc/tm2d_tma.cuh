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
// Warp roles.  A CTA has 16 compute warps and one producer warp.  The
// producer walks the CTA's units kQStages ahead of the compute warps: for
// each it waits until the stage is empty (an mbarrier the compute warps
// arrive on), stages the tile's point entries (cell, value) and -- on a new
// tile -- its CPML profile values into shared memory, then issues 3-D tiled
// TMA loads of the three fields (with the halo) and, on a new tile, of the
// model coefficients, all completing on the stage's full mbarrier.  The
// compute warps therefore never issue a transfer and never wait on a
// dependent global load for profile values or point lists; elements outside
// the grid read as zero.  Results go back with coalesced stores; snapshots
// (caller layout, rows of nx cells at any alignment) with streaming scalar
// stores / loads, the adjoint's loaded one unit ahead.
//
// Layout of the work.  A tile is 32 rows x 64 columns; compute warp w owns
// rows 2w and 2w+1 of it, lane l the columns l and l + 32, so every shared
// memory access of a warp is 32 consecutive words (no bank conflict) and
// every store 128 contiguous bytes.
//
// Schedule.  The grid is persistent: P CTAs (one per SM; P <= tiles), CTA c
// owns the units [c U / P, (c+1) U / P) of the tile-major sequence of
// U = tiles x shots (tile, shot) units, so every CTA gets the same number of
// units to within one.  The tile sequence is a host-chosen permutation that
// spreads the tiles with CPML strips or grid edges (the slower ones) evenly
// over it, so every CTA gets the same mix.  A tile's shots are processed in
// ascending order, so the adjoint's coefficient gradient is the kernels'
// step-major shot sum (grad += ((0 + t_0) + t_1) + ...), bit-identical to
// the other stencil-2 kernels and to the oracle in that order.  A tile whose
// shots are split between CTA c-1 (shots [0, k), processed first) and CTA c
// (shots [k, S), processed last) hands the running sums over through global
// memory: CTA c-1 stores them and releases a flag, CTA c acquires it (a
// bounded wait, normally long satisfied) and continues the sums.
//
// Numerics.  Every cell value is computed with the same operations in the
// same order as tm2d_s2.cuh (--fmad=false), so fields, snapshots, receivers,
// source gradients and the model gradient are bit-identical to that path.
#pragma once

#include "tb_tma.cuh"
#include "tm2d_kernels.cuh"

namespace tb {

constexpr int kQX = 64;                          // tile width (cells)
constexpr int kQTY_ = 32;                        // tile height (cells)
constexpr int kQCWarps = 16;                     // compute warps
constexpr int kQCompute = 32 * kQCWarps;         // compute threads
constexpr int kQThreads = kQCompute + 32;        // + the producer warp
constexpr int kQStages = 3;                      // units in flight
constexpr int kQPtCap = 64;                      // point entries staged per list
constexpr uint32_t kQWaitLimit = 1u << 24;       // bounded waits (polls)
constexpr int kQPW = kQX + 2;                    // profile columns x0-1 .. x0+64
constexpr int kQPH = kQTY_ + 2;                  // profile rows y0-1 .. y0+32

// Bytes rounded up to the 128-byte alignment of every shared-memory buffer.
constexpr int q_rb(int bytes) { return (bytes + 127) / 128 * 128; }

// Shared-memory extents (floats) of the staged boxes.
struct QBox {
  static constexpr int TY = kQTY_;
  static constexpr int EW = kQX + 8, EH = TY + 2;  // rows y0-1..y0+TY,   cols x0-4..x0+67
  static constexpr int XW = kQX, XH = TY + 1;      // rows y0-1..y0+TY-1, cols x0..x0+63
  static constexpr int ZW = kQX + 4, ZH = TY;      // rows y0..y0+TY-1,   cols x0-4..x0+63
  static constexpr int OW = kQX, OH = TY;          // own cells
  static constexpr int QW = kQX + 4, QH = TY + 1;  // rows y0-1..y0+TY-1, cols x0-4..x0+63
  static constexpr int E_B = q_rb(4 * EW * EH), X_B = q_rb(4 * XW * XH),
                       Z_B = q_rb(4 * ZW * ZH), O_B = q_rb(4 * OW * OH), Q_B = q_rb(4 * QW * QH);
  // staged point lists: counts (2 ints) then list A (index, value) and list B
  // (index, entry), kQPtCap each
  static constexpr int PT_B = q_rb(4 * (2 + 4 * kQPtCap));
  // CPML profiles of a tile: x (bx ax kx bxh axh kxh) x kQPW, y (by ay ky byh ayh kyh) x kQPH
  static constexpr int PR_B = q_rb(4 * 6 * (kQPW + kQPH));
  static constexpr int STAGE_B = E_B + X_B + Z_B + PT_B;
  static constexpr int COEF_ADJ_B = O_B + E_B + Q_B + PR_B;  // ca, cb (E box), cq (Q box)
  static constexpr int COEF_FWD_B = Q_B + O_B + O_B + PR_B;  // cq (Q box), ca, cb
  static constexpr int EXTRA_B = X_B + Z_B;                   // new Hx, new Hz
  static constexpr int smem_bytes(bool adj) {
    return kQStages * (STAGE_B + (adj ? COEF_ADJ_B : COEF_FWD_B)) + EXTRA_B +
           16 * kQStages;
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
// between at most two CTAs.  Tiles are positions in the tile sequence.
struct QSched {
  int S;
  int nA, nB, nC;
  int tA, tB0, tC, cC0;
  __device__ __forceinline__ int n() const { return nA + nB + nC; }
  // (sequence tile, shot, ordinal of the tile in this CTA's sequence, segment 0/1/2)
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

// Shared memory carve-up: kQStages stages (fields + point lists),
// kQStages coefficient slots (coefficients + profiles), the new-H tiles and
// the full / empty barriers of the stages.  Addresses are computed, not
// tabulated, so nothing is indexed dynamically in local memory.
template <bool ADJ> struct QSmem {
  using B = QBox;
  static constexpr int COEF_B = ADJ ? B::COEF_ADJ_B : B::COEF_FWD_B;
  static constexpr int COEF0 = kQStages * B::STAGE_B;
  static constexpr int EXTRA0 = COEF0 + kQStages * COEF_B;
  unsigned char *base;
  float *hxn, *hzn;
  uint64_t *full, *empty;
  __device__ __forceinline__ explicit QSmem(unsigned char *b) : base(b) {
    hxn = reinterpret_cast<float *>(b + EXTRA0);
    hzn = reinterpret_cast<float *>(b + EXTRA0 + B::X_B);
    full = reinterpret_cast<uint64_t *>(b + EXTRA0 + B::EXTRA_B);
    empty = full + kQStages;
  }
  __device__ __forceinline__ unsigned char *st(int k) const { return base + k * B::STAGE_B; }
  __device__ __forceinline__ float *e(int k) const { return reinterpret_cast<float *>(st(k)); }
  __device__ __forceinline__ float *x(int k) const {
    return reinterpret_cast<float *>(st(k) + B::E_B);
  }
  __device__ __forceinline__ float *z(int k) const {
    return reinterpret_cast<float *>(st(k) + B::E_B + B::X_B);
  }
  __device__ __forceinline__ int *pt(int k) const {
    return reinterpret_cast<int *>(st(k) + B::E_B + B::X_B + B::Z_B);
  }
  __device__ __forceinline__ unsigned char *cs(int k) const {
    return base + COEF0 + k * COEF_B;
  }
  // adjoint: c0 = ca (own box), c1 = cb (E box), c2 = cq (Q box);
  // forward: c0 = cq (Q box), c1 = ca (own box), c2 = cb (own box)
  __device__ __forceinline__ float *c0(int k) const { return reinterpret_cast<float *>(cs(k)); }
  __device__ __forceinline__ float *c1(int k) const {
    return reinterpret_cast<float *>(cs(k) + (ADJ ? B::O_B : B::Q_B));
  }
  __device__ __forceinline__ float *c2(int k) const {
    return reinterpret_cast<float *>(cs(k) + (ADJ ? B::O_B + B::E_B : B::Q_B + B::O_B));
  }
  __device__ __forceinline__ float *pr(int k) const {
    return reinterpret_cast<float *>(cs(k) + COEF_B - B::PR_B);
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
  const int *order;           // grid tile at each position of the tile sequence
  int64_t pitch, pshot;       // floats per pitched row / per pitched shot
  float *ey_n, *hx_n, *hz_n;  // next copy (pitched)
  PointCSR pa, pb;            // list A (values added) / list B (values recorded):
                              // forward sources / receivers, adjoint receivers / sources
  const float *va;            // forward: f_t; adjoint: grad_r_t
  float *vb;                  // forward: r_t; adjoint: grad_f_t
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
  float *hand;  // [P][2][32 * 64] running sums handed from CTA c-1 to c
  int *flags;   // [P]
  int epoch;    // distinct per launch within a call (flags start at 0)
};

// Compute-warp barrier (the producer warp does not take part).
__device__ __forceinline__ void q_csync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kQCompute) : "memory");
}

// Tile-local index (oy * 64 + ox) of a flat cell, or -1 outside the tile.
__device__ __forceinline__ int q_local(int cell, int ybase, int nx) {
  const int d = cell - ybase;
  if (d < 0) return -1;
  const int oy = d / nx, ox = d - oy * nx;
  return (oy < kQTY_ && ox < kQX) ? oy * kQX + ox : -1;
}

// ------------------------------------------------------------ producer

// Stage one point list of unit pid into dst: count (or -1 when it holds
// more than kQPtCap entries), then (local index, value / entry) pairs in
// entry order.  Executed by the 32 lanes of the producer warp.
__device__ __forceinline__ void q_stage_list(const PointCSR &pl, const float *vals, bool by_value,
                                             int pid, int ybase, int nx, int *cnt, int *dst) {
  const int lane = threadIdx.x & 31;
  int n = 0;
  if (pl.start != nullptr && vals != nullptr) {
    const int b = __ldg(pl.start + pid), e = __ldg(pl.start + pid + 1);
    n = e - b;
    if (n > kQPtCap) {
      n = -1;
    } else {
      for (int i = lane; i < n; i += 32) {
        const int ent = __ldg(pl.ent + b + i);
        dst[2 * i] = q_local(__ldg(pl.cell + b + i), ybase, nx);
        dst[2 * i + 1] = by_value ? __float_as_int(__ldg(vals + ent)) : ent;
      }
    }
  }
  if (lane == 0) *cnt = n;
}

// Profiles of a new tile: x profiles at columns x0-1 .. x0+64 and y profiles
// at rows y0-1 .. y0+32 (zero, kappa one, outside the grid).
__device__ __forceinline__ void q_stage_profiles(const TMGeom<float> &g, int y0, int x0,
                                                 float *pr) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < 6 * kQPW; i += 32) {
    const int a = i / kQPW, c = i - a * kQPW, x = x0 - 1 + c;
    const float *p = a == 0 ? g.bx : a == 1 ? g.ax : a == 2 ? g.kx
                   : a == 3 ? g.bxh : a == 4 ? g.axh : g.kxh;
    pr[i] = (x >= 0 && x < g.nx) ? __ldg(p + x) : ((a == 2 || a == 5) ? 1.f : 0.f);
  }
  for (int i = lane; i < 6 * kQPH; i += 32) {
    const int a = i / kQPH, r = i - a * kQPH, y = y0 - 1 + r;
    const float *p = a == 0 ? g.by : a == 1 ? g.ay : a == 2 ? g.ky
                   : a == 3 ? g.byh : a == 4 ? g.ayh : g.kyh;
    pr[6 * kQPW + i] = (y >= 0 && y < g.ny) ? __ldg(p + y) : ((a == 2 || a == 5) ? 1.f : 0.f);
  }
}

// The producer warp: for every unit of the CTA (kQStages ahead of the
// compute warps) wait for the stage to be empty, stage point lists and, on a
// new tile, profiles, then lane 0 issues the TMA loads on the full barrier.
template <bool ADJ>
__device__ __forceinline__ void q_producer(const QSmem<ADJ> &sm, const QMaps &m,
                                           const QCommon &cm, const QSched &sc) {
  using B = QBox;
  const int lane = threadIdx.x & 31;
  const TMGeom<float> &g = cm.g;
  const int n_units = sc.n();
  int prev_ord = -1;
  for (int j = 0; j < n_units; ++j) {
    const int k = j % kQStages;
    if (j >= kQStages &&
        !mbar_wait(sm.empty + k, (uint32_t)((j / kQStages - 1) & 1), kQWaitLimit) &&
        lane == 0)
      atomicOr(&g_tide_dev_err, 16);
    int stile, shot, ord, seg;
    sc.unit(j, stile, shot, ord, seg);
    const int tile = __ldg(cm.order + stile);
    const int ty = tile / cm.tiles_x, tx = tile - ty * cm.tiles_x;
    const int y0 = ty * B::TY, x0 = tx * kQX;
    const bool new_tile = ord != prev_ord;
    prev_ord = ord;
    const int cs = ord % kQStages;
    // point lists of (tile, shot)
    const int pid = (shot * cm.tiles_y + ty) * cm.tiles_x + tx;
    int *pt = sm.pt(k);
    q_stage_list(cm.pa, cm.va, true, pid, y0 * g.nx + x0, g.nx, pt, pt + 2);
    q_stage_list(cm.pb, cm.vb, false, pid, y0 * g.nx + x0, g.nx, pt + 1, pt + 2 + 2 * kQPtCap);
    if (new_tile) q_stage_profiles(g, y0, x0, sm.pr(cs));
    __syncwarp();
    if (lane == 0) {
      uint64_t *bar = sm.full + k;
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(
          bar, B::FIELD_TX + (new_tile ? (ADJ ? B::COEF_ADJ_TX : B::COEF_FWD_TX) : 0u));
      tma_load_3d(sm.e(k), &m.e, bar, x0 - 4, y0 - 1, shot);
      tma_load_3d(sm.x(k), &m.x, bar, x0, y0 - 1, shot);
      tma_load_3d(sm.z(k), &m.z, bar, x0 - 4, y0, shot);
      if (new_tile) {
        if (ADJ) {
          tma_load_3d(sm.c0(cs), &m.c0, bar, x0, y0, 0);
          tma_load_3d(sm.c1(cs), &m.c1, bar, x0 - 4, y0 - 1, 0);
          tma_load_3d(sm.c2(cs), &m.c2, bar, x0 - 4, y0 - 1, 0);
        } else {
          tma_load_3d(sm.c0(cs), &m.c0, bar, x0 - 4, y0 - 1, 0);
          tma_load_3d(sm.c1(cs), &m.c1, bar, x0, y0, 0);
          tma_load_3d(sm.c2(cs), &m.c2, bar, x0, y0, 0);
        }
      }
    }
  }
}

// Barrier set-up and tensor-map prefetch (thread 0), then a block barrier.
template <bool ADJ>
__device__ __forceinline__ void q_setup(const QSmem<ADJ> &sm, const QMaps &m) {
  if (threadIdx.x == 0) {
    for (int k = 0; k < kQStages; ++k) {
      mbar_init(sm.full + k, 1);
      mbar_init(sm.empty + k, kQCWarps);
    }
    mbar_init_fence();
    tma_prefetch_map(&m.e);
    tma_prefetch_map(&m.x);
    tma_prefetch_map(&m.z);
    tma_prefetch_map(&m.c0);
    tma_prefetch_map(&m.c1);
    tma_prefetch_map(&m.c2);
  }
  __syncthreads();
}

// ------------------------------------------------------------ compute helpers

// Profile lookups in a tile's staged profiles.
struct QProf {
  const float *p;
  int x0, y0;
  // a: 0 b, 1 a, 2 kappa (integer grid), 3 bh, 4 ah, 5 kappah (half grid)
  __device__ __forceinline__ float x(int a, int xx) const { return p[a * kQPW + xx - x0 + 1]; }
  __device__ __forceinline__ float y(int a, int yy) const {
    return p[6 * kQPW + a * kQPH + yy - y0 + 1];
  }
};

// Point passes over the own cells (values v[r][q] at rows 2w + r, columns
// l + 32 q) from the staged lists; a list that did not fit the stage is read
// from global memory instead.  Entries at one cell are applied in entry order.
__device__ __forceinline__ void q_points(const int *pt, const QCommon &cm, int pid, int ybase,
                                         float (&v)[2][2]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int na = pt[0], nb = pt[1];
  const int *la = pt + 2, *lb = pt + 2 + 2 * kQPtCap;
  if (na != 0) {
    int b = 0, e = 0;
    if (na < 0) {
      b = __ldg(cm.pa.start + pid);
      e = __ldg(cm.pa.start + pid + 1);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int me = (2 * warp + r) * kQX + lane + 32 * q;
        if (na > 0) {
          for (int i = 0; i < na; ++i)
            if (la[2 * i] == me) v[r][q] = v[r][q] + __int_as_float(la[2 * i + 1]);
        } else {
          for (int i = b; i < e; ++i)
            if (q_local(__ldg(cm.pa.cell + i), ybase, cm.g.nx) == me)
              v[r][q] = v[r][q] + __ldg(cm.va + __ldg(cm.pa.ent + i));
        }
      }
  }
  if (nb != 0) {
    int b = 0, e = 0;
    if (nb < 0) {
      b = __ldg(cm.pb.start + pid);
      e = __ldg(cm.pb.start + pid + 1);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int me = (2 * warp + r) * kQX + lane + 32 * q;
        if (nb > 0) {
          for (int i = 0; i < nb; ++i)
            if (lb[2 * i] == me) cm.vb[lb[2 * i + 1]] = v[r][q];
        } else {
          for (int i = b; i < e; ++i)
            if (q_local(__ldg(cm.pb.cell + i), ybase, cm.g.nx) == me)
              cm.vb[__ldg(cm.pb.ent + i)] = v[r][q];
        }
      }
  }
}

// CPML memory values one cell reads (loaded before its arithmetic, so a
// strip tile waits for memory once per phase, not once per cell).
struct QM4 {
  float a, b, c, d;
};

// Interior tile: no cell it updates or recomputes is in a CPML strip or on
// the grid edge.
__device__ __forceinline__ bool q_interior(const TMGeom<float> &g, int y0, int x0) {
  return y0 - 1 >= max(1, g.pml_y0) && y0 + kQTY_ < min(g.ny, g.pml_y1) &&
         x0 - 1 >= max(1, g.pml_x0) && x0 + kQX < min(g.nx, g.pml_x1);
}

// ============================================================== adjoint
//
// Per unit: phase 1 = adjoint E-phase (cb lEy -> lHx, lHz and the E-phase
// memories) on the own cells plus the halo row y0-1 (lHx) and column x0-1
// (lHz), into shared memory; phase 2 = adjoint H-phase (lEy from the new
// lHx / lHz, the H-phase memories), receivers injected, sources recorded,
// image terms summed over the tile's shots.  Formulas: tm2d_s2.cuh
// adj_e_tile / adj_h_tile.
struct QAdjCell {
  using B = QBox;
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
  static __device__ __forceinline__ void e_phase(const QAdjArgs &a, const QProf &pf,
                                                 const float *E, const float *CB, float lhx,
                                                 float lhz, int y, int x, int y0, int x0,
                                                 int64_t sb, bool own, const QM4 &m,
                                                 float &hx_new, float &hz_new) {
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
      const float mn = pf.x(0, x) * m.a + q;
      rx = pf.x(1, x) * mn + q / pf.x(2, x);
      if (own) a.mhz_n[j] = mn;
    }
    if (x + 1 >= g.nx) {
      rxr = 0.f;
    } else if (!xs(g, x + 1)) {
      rxr = qr;
    } else {
      const float mn = pf.x(0, x + 1) * m.b + qr;
      rxr = pf.x(1, x + 1) * mn + qr / pf.x(2, x + 1);
    }
    if (!ys(g, y)) {
      ry0 = -q;
    } else {
      const float mn = pf.y(0, y) * m.c - q;
      ry0 = pf.y(1, y) * mn - q / pf.y(2, y);
      if (own) a.mhx_n[j] = mn;
    }
    if (y + 1 >= g.ny) {
      ry1 = 0.f;
    } else if (!ys(g, y + 1)) {
      ry1 = -q1;
    } else {
      const float mn = pf.y(0, y + 1) * m.d - q1;
      ry1 = pf.y(1, y + 1) * mn - q1 / pf.y(2, y + 1);
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
  static __device__ __forceinline__ float h_phase(const QAdjArgs &a, const QProf &pf,
                                                  const float *E, const float *CA,
                                                  const float *CQ, const float *HXN,
                                                  const float *HZN, int y, int x, int y0, int x0,
                                                  int64_t sb, const QM4 &m) {
    const TMGeom<float> &g = a.c.g;
    const int oy = y - y0, ox = x - x0;
    const float lam = E[(oy + 1) * B::EW + ox + 4];
    const float ca = CA[oy * B::OW + ox];
    const float cz0 = CQ[oy * B::QW + ox + 4], cz1 = CQ[(oy + 1) * B::QW + ox + 4];
    const float cl = CQ[(oy + 1) * B::QW + ox + 3];
    const float h0 = HXN[oy * B::XW + ox], h1 = HXN[(oy + 1) * B::XW + ox];
    const float zx = HZN[oy * B::ZW + ox + 4], zl = HZN[oy * B::ZW + ox + 3];
    if (IN) {
      const float rz0 = -cz0 * h0, rz1 = -cz1 * h1;
      const float rx = cz1 * zx, rxl = cl * zl;
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
          const float mn = pf.y(3, yy) * m.a + adj;
          rz0 = pf.y(4, yy) * mn + adj / pf.y(5, yy);
        }
      }
    }
    if (y < g.ny - 1) {  // row y (y >= 1 here)
      const float adj = -cz1 * h1;
      if (!ysh(g, y)) {
        rz1 = adj;
      } else {
        const float mn = pf.y(3, y) * m.b + adj;
        rz1 = pf.y(4, y) * mn + adj / pf.y(5, y);
        a.mez_n[j] = mn;
      }
    }
    if (x < g.nx - 1) {  // column x (x >= 1 here)
      const float adj = cz1 * zx;
      if (!xsh(g, x)) {
        rx = adj;
      } else {
        const float mn = pf.x(3, x) * m.c + adj;
        rx = pf.x(4, x) * mn + adj / pf.x(5, x);
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
          const float mn = pf.x(3, xl) * m.d + adj;
          rxl = pf.x(4, xl) * mn + adj / pf.x(5, xl);
        }
      }
    }
    float v = ca * lam;
    v = v + (((float)1 * (rz0 - rz1)) * g.rdy + ((float)1 * (rxl - rx)) * g.rdx);
    return v;
  }
};

template <typename SN> __device__ __forceinline__ float q_dec(SN v) { return Codec<SN, float>::dec(v); }

// Snapshots of the own cells of unit (grid tile, shot): shot s images
// against snapshot shot s % bg_shots; cells outside the update domain read
// nothing.
template <typename SN>
__device__ __forceinline__ void q_snap_load(const QAdjArgs &a, int tile, int shot,
                                            SN (&ev)[2][2], SN (&cv)[2][2]) {
  const TMGeom<float> &g = a.c.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ty = tile / a.c.tiles_x;
  const int y0 = ty * kQTY_, x0 = (tile - ty * a.c.tiles_x) * kQX;
  const int64_t snb = (int64_t)(shot % a.bg_shots) * g.N;
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int y = y0 + 2 * warp + r, x = x0 + lane + 32 * q;
      const bool ok = y >= 1 && x >= 1 && y < g.ny && x < g.nx;
      const int64_t j = snb + (int64_t)y * g.nx + x;
      ev[r][q] = (ok && a.ey_st) ? load_stream(static_cast<const SN *>(a.ey_st) + j) : SN(0.f);
      cv[r][q] = (ok && a.cu_st) ? load_stream(static_cast<const SN *>(a.cu_st) + j) : SN(0.f);
    }
}

template <typename SN>
__global__ void __launch_bounds__(kQThreads, 1)
kq_adj_step(const __grid_constant__ QMaps m, const QAdjArgs a) {
  using B = QBox;
  using C = QAdjCell;
  extern __shared__ __align__(128) unsigned char q_smem[];
  const QSmem<true> sm(q_smem);
  const QCommon &cm = a.c;
  const TMGeom<float> &g = cm.g;
  const int S = g.n_shots, nx = g.nx, ny = g.ny;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cta = blockIdx.x;
  const QSched sc = q_sched(cta, cm.P, cm.tiles_x * cm.tiles_y, S);
  const int n_units = sc.n();
  const bool imaging = a.ey_st != nullptr || a.cu_st != nullptr;

  q_setup<true>(sm, m);
  if (warp == kQCWarps) {
    q_producer<true>(sm, m, cm, sc);
    return;
  }

  float sum_a[2][2], sum_b[2][2];
  // snapshots are loaded one unit ahead (their latency overlaps a whole unit)
  SN ev[2][2], cv[2][2];
  if (imaging && n_units > 0) {
    int t0, s0, o0, g0;
    sc.unit(0, t0, s0, o0, g0);
    q_snap_load<SN>(a, __ldg(cm.order + t0), s0, ev, cv);
  }
  const QM4 z4{0.f, 0.f, 0.f, 0.f};
  int prev_ord = -1;
  for (int i = 0; i < n_units; ++i) {
    int stile, shot, ord, seg;
    sc.unit(i, stile, shot, ord, seg);
    const int tile = __ldg(cm.order + stile);
    const int k = i % kQStages;
    const int cs = ord % kQStages;
    const int ty = tile / cm.tiles_x, tx = tile - ty * cm.tiles_x;
    const int y0 = ty * B::TY, x0 = tx * kQX;
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
        q_csync();
        const float *h = a.hand + (size_t)(cta - 1) * 2 * B::TY * kQX;
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int o = (2 * warp + r) * kQX + lane + 32 * q;
            sum_a[r][q] = __ldcg(h + o);
            sum_b[r][q] = __ldcg(h + B::TY * kQX + o);
          }
      } else {
#pragma unroll
        for (int r = 0; r < 2; ++r) sum_a[r][0] = sum_a[r][1] = sum_b[r][0] = sum_b[r][1] = 0.f;
      }
    }
    SN evn[2][2], cvn[2][2];
    if (imaging && i + 1 < n_units) {
      int t1, s1, o1, g1;
      sc.unit(i + 1, t1, s1, o1, g1);
      q_snap_load<SN>(a, __ldg(cm.order + t1), s1, evn, cvn);
    }
    // A transfer that never lands ends the wait with the error word set; the
    // CTA still runs every barrier so the launch finishes.
    if (!mbar_wait(sm.full + k, (uint32_t)((i / kQStages) & 1), kQWaitLimit))
      atomicOr(&g_tide_dev_err, 8);
    const float *E = sm.e(k), *LX = sm.x(k), *LZ = sm.z(k);
    const float *CA = sm.c0(cs), *CB = sm.c1(cs), *CQ = sm.c2(cs);
    const QProf pf{sm.pr(cs), x0, y0};
    const bool in = q_interior(g, y0, x0);
    // ---------------- phase 1: adjoint E-phase
    // (strip tiles: every memory value the thread's cells read is loaded first)
    QM4 mm[2][2], mh[2];
    if (!in) {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::e_loads(a, y0 + 2 * warp + r, x0 + lane + 32 * q, sb);
      if (warp == 0) {
        mh[0] = C::e_loads(a, y0 - 1, x0 + lane, sb);
        mh[1] = C::e_loads(a, y0 - 1, x0 + lane + 32, sb);
      } else if (warp == 1) {
        mh[0] = C::e_loads(a, y0 + lane, x0 - 1, sb);
      }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int oy = 2 * warp + r, y = y0 + oy;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = lane + 32 * q, x = x0 + ox;
        const float lhx = LX[(oy + 1) * B::XW + ox], lhz = LZ[oy * B::ZW + ox + 4];
        float hxn, hzn;
        if (in)
          C::e_phase<true>(a, pf, E, CB, lhx, lhz, y, x, y0, x0, sb, true, z4, hxn, hzn);
        else
          C::e_phase<false>(a, pf, E, CB, lhx, lhz, y, x, y0, x0, sb, true, mm[r][q], hxn, hzn);
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
        const int ox = lane + 32 * q, y = y0 - 1, x = x0 + ox;
        float hxn, hzn;
        if (in)
          C::e_phase<true>(a, pf, E, CB, LX[ox], 0.f, y, x, y0, x0, sb, false, z4, hxn, hzn);
        else
          C::e_phase<false>(a, pf, E, CB, LX[ox], 0.f, y, x, y0, x0, sb, false, mh[q], hxn,
                            hzn);
        sm.hxn[ox] = hxn;
      }
    } else if (warp == 1) {  // halo column x0 - 1 (new lHz only)
      const int oy = lane, y = y0 + oy, x = x0 - 1;
      const float lhz = LZ[oy * B::ZW + 3];
      float hxn, hzn;
      if (in)
        C::e_phase<true>(a, pf, E, CB, 0.f, lhz, y, x, y0, x0, sb, false, z4, hxn, hzn);
      else
        C::e_phase<false>(a, pf, E, CB, 0.f, lhz, y, x, y0, x0, sb, false, mh[0], hxn, hzn);
      sm.hzn[oy * B::ZW + 3] = hzn;
    }
    q_csync();
    // ---------------- phase 2: adjoint H-phase
    float v[2][2];
    if (in) {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          v[r][q] = C::h_phase<true>(a, pf, E, CA, CQ, sm.hxn, sm.hzn, y0 + 2 * warp + r,
                                     x0 + lane + 32 * q, y0, x0, sb, z4);
    } else {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::h_loads(a, y0 + 2 * warp + r, x0 + lane + 32 * q, sb);
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          v[r][q] = C::h_phase<false>(a, pf, E, CA, CQ, sm.hxn, sm.hzn, y0 + 2 * warp + r,
                                      x0 + lane + 32 * q, y0, x0, sb, mm[r][q]);
    }
    // receivers (lEy += grad_r, entry order), then sources (grad_f = lEy)
    const int pid = (shot * cm.tiles_y + ty) * cm.tiles_x + tx;
    q_points(sm.pt(k), cm, pid, y0 * nx + x0, v);
    // the stage (fields, point lists) is no longer read by this warp
    __syncwarp();
    if (lane == 0) mbar_arrive(sm.empty + k);
    // store lEy, image terms
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int y = y0 + 2 * warp + r;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int x = x0 + lane + 32 * q;
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
        float *h = a.hand + (size_t)cta * 2 * B::TY * kQX;
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int o = (2 * warp + r) * kQX + lane + 32 * q;
            __stcg(h + o, sum_a[r][q]);
            __stcg(h + B::TY * kQX + o, sum_b[r][q]);
          }
        __threadfence();
        q_csync();
        if (tid == 0) st_release_gpu(a.flags + cta, a.epoch);
      } else {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int y = y0 + 2 * warp + r;
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int x = x0 + lane + 32 * q;
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
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        ev[r][q] = evn[r][q];
        cv[r][q] = cvn[r][q];
      }
    q_csync();  // the new-H tiles are free for the next unit
  }
}

// ============================================================== forward
//
// Per unit: phase 1 = H half step (new Hx on rows y0-1..y0+31, new Hz on
// columns x0-1..x0+63; own cells write the next H-phase memories), phase 2 =
// E half step on the own cells (E-phase memories in place), snapshots of
// Ey^n and curl H, sources added, receivers recorded.  Formulas:
// tm2d_s2.cuh fwd_h_tile / fwd_e_tile.
struct QFwdCell {
  using B = QBox;
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
  static __device__ __forceinline__ void h_phase(const QFwdArgs &a, const QProf &pf,
                                                 const float *E, const float *CQ, float hx,
                                                 float hz, int y, int x, int y0, int x0,
                                                 int64_t sb, bool own, const QM4 &m,
                                                 float &hx_new, float &hz_new) {
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
        const float mm = pf.y(3, y) * m.a + pf.y(4, y) * d;
        if (own) a.mez_n[j] = mm;
        d = d / pf.y(5, y) + mm;
      }
      hx_new = hx - c * d;
    }
    if (x < g.nx - 1) {
      float d = (er - e0) * g.rdx;
      if (x < g.pml_x0 || x >= g.pml_x1h) {
        const float mm = pf.x(3, x) * m.b + pf.x(4, x) * d;
        if (own) a.mex_n[j] = mm;
        d = d / pf.x(5, x) + mm;
      }
      hz_new = hz + c * d;
    }
  }
};

template <typename SN>
__global__ void __launch_bounds__(kQThreads, 1)
kq_fwd_step(const __grid_constant__ QMaps m, const QFwdArgs a) {
  using B = QBox;
  using C = QFwdCell;
  extern __shared__ __align__(128) unsigned char q_smem[];
  const QSmem<false> sm(q_smem);
  const QCommon &cm = a.c;
  const TMGeom<float> &g = cm.g;
  const int nx = g.nx, ny = g.ny;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const QSched sc = q_sched(blockIdx.x, cm.P, cm.tiles_x * cm.tiles_y, g.n_shots);
  const int n_units = sc.n();

  q_setup<false>(sm, m);
  if (warp == kQCWarps) {
    q_producer<false>(sm, m, cm, sc);
    return;
  }
  const QM4 z4{0.f, 0.f, 0.f, 0.f};
  for (int i = 0; i < n_units; ++i) {
    int stile, shot, ord, seg;
    sc.unit(i, stile, shot, ord, seg);
    const int tile = __ldg(cm.order + stile);
    const int k = i % kQStages;
    const int cs = ord % kQStages;
    const int ty = tile / cm.tiles_x, tx = tile - ty * cm.tiles_x;
    const int y0 = ty * B::TY, x0 = tx * kQX;
    const int64_t sb = (int64_t)shot * g.N;
    const int64_t pb = (int64_t)shot * cm.pshot;
    if (!mbar_wait(sm.full + k, (uint32_t)((i / kQStages) & 1), kQWaitLimit))
      atomicOr(&g_tide_dev_err, 8);
    const float *E = sm.e(k), *HX = sm.x(k), *HZ = sm.z(k);
    const float *CQ = sm.c0(cs), *CA = sm.c1(cs), *CB = sm.c2(cs);
    const QProf pf{sm.pr(cs), x0, y0};
    const bool in = q_interior(g, y0, x0);
    // ---------------- phase 1: H half step
    // (strip tiles: the memories of the thread's cells are loaded first)
    QM4 mm[2][2], mh[2];
    if (!in) {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::h_loads(a, y0 + 2 * warp + r, x0 + lane + 32 * q, sb);
      if (warp == 0) {
        mh[0] = C::h_loads(a, y0 - 1, x0 + lane, sb);
        mh[1] = C::h_loads(a, y0 - 1, x0 + lane + 32, sb);
      } else if (warp == 1) {
        mh[0] = C::h_loads(a, y0 + lane, x0 - 1, sb);
      }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int oy = 2 * warp + r, y = y0 + oy;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = lane + 32 * q, x = x0 + ox;
        const float hx = HX[(oy + 1) * B::XW + ox], hz = HZ[oy * B::ZW + ox + 4];
        float hxn, hzn;
        if (in)
          C::h_phase<true>(a, pf, E, CQ, hx, hz, y, x, y0, x0, sb, true, z4, hxn, hzn);
        else
          C::h_phase<false>(a, pf, E, CQ, hx, hz, y, x, y0, x0, sb, true, mm[r][q], hxn, hzn);
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
        const int ox = lane + 32 * q;
        float hxn, hzn;
        if (in)
          C::h_phase<true>(a, pf, E, CQ, HX[ox], 0.f, y0 - 1, x0 + ox, y0, x0, sb, false, z4,
                           hxn, hzn);
        else
          C::h_phase<false>(a, pf, E, CQ, HX[ox], 0.f, y0 - 1, x0 + ox, y0, x0, sb, false, mh[q],
                            hxn, hzn);
        sm.hxn[ox] = hxn;
      }
    } else if (warp == 1) {  // halo column x0 - 1 (new Hz only)
      const int oy = lane;
      float hxn, hzn;
      if (in)
        C::h_phase<true>(a, pf, E, CQ, 0.f, HZ[oy * B::ZW + 3], y0 + oy, x0 - 1, y0, x0, sb,
                         false, z4, hxn, hzn);
      else
        C::h_phase<false>(a, pf, E, CQ, 0.f, HZ[oy * B::ZW + 3], y0 + oy, x0 - 1, y0, x0, sb,
                          false, mh[0], hxn, hzn);
      sm.hzn[oy * B::ZW + 3] = hzn;
    }
    q_csync();
    // ---------------- phase 2: E half step
    float v[2][2];
    if (!in) {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int q = 0; q < 2; ++q)
          mm[r][q] = C::e_loads(a, y0 + 2 * warp + r, x0 + lane + 32 * q, sb);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int oy = 2 * warp + r, y = y0 + oy;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int ox = lane + 32 * q, x = x0 + ox;
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
            const float m1 = pf.x(0, x) * mm[r][q].a + pf.x(1, x) * dz;
            a.mhz[j] = m1;
            dz = dz / pf.x(2, x) + m1;
          }
          if (y < g.pml_y0 || y >= g.pml_y1) {
            const float m1 = pf.y(0, y) * mm[r][q].b + pf.y(1, y) * dy;
            a.mhx[j] = m1;
            dy = dy / pf.y(2, y) + m1;
          }
          const float curl = dz - dy;
          if (a.ey_st) store_stream(static_cast<SN *>(a.ey_st) + j, Codec<SN, float>::enc(eo));
          if (a.cu_st) store_stream(static_cast<SN *>(a.cu_st) + j, Codec<SN, float>::enc(curl));
          e = ca * eo + cb * curl;
        }
        v[r][q] = e;
      }
    }
    // sources (Ey += f, entry order), then receivers (r = Ey)
    const int pid = (shot * cm.tiles_y + ty) * cm.tiles_x + tx;
    q_points(sm.pt(k), cm, pid, y0 * nx + x0, v);
    __syncwarp();
    if (lane == 0) mbar_arrive(sm.empty + k);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int y = y0 + 2 * warp + r;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int x = x0 + lane + 32 * q;
        if (y < ny && x < nx) cm.ey_n[pb + (int64_t)y * cm.pitch + x] = v[r][q];
      }
    }
    q_csync();  // the new-H tiles are free for the next unit
  }
}

}  // namespace tb
