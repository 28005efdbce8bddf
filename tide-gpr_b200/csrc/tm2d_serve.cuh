// Multi-job TM2D serving engine (stencil order 2, float32); interface in
// include/tide_b200_serve.h.
//
// Design.  Every resident job ("slot") keeps its coefficients, state, CPML
// memories, adjoint fields and tile lists in device memory for its whole
// life.  A chunk of C time steps is four kernel chains per step: forward H and
// forward E over the tiles of all slots in a forward phase, adjoint E and
// adjoint H over the tiles of all slots in the adjoint phase.  The forward
// and adjoint chains touch disjoint slots, so they run on two streams (two
// independent branches of the chunk's CUDA graph) and overlap.  Each kernel
// is persistent: a grid of (SMs x resident CTAs) walks the virtual tiles of
// the chunk's work table (prefix sums of tile counts per slot and kernel
// kind), so the launch parameters do not depend on the job mix and one
// captured graph per chunk length serves every chunk.  A CTA maps its tile
// to (slot, tile x, tile y, shot) and runs the per-call kernels' tile
// function on it, so each cell of each job is computed exactly as in the
// per-call path.
//
// The work table (geometry, pointers, phase, first step, steps this chunk,
// snapshot bases) is built on the host before each chunk in pinned memory and
// copied to the device on the engine's stream ahead of the chunk's kernels.
//
// Large slots (shots x cells at or above the engine's direct threshold) do
// not go through the table: their tiles fill the GPU on their own, and the
// per-call kernels (parameters in the constant bank, fewer registers, and the
// fused pitched forward step) are faster per cell than the table walk.  Each
// runs its steps with the per-call launches on one of a pool of streams,
// concurrently with the table chains and with the other large slots.  A
// large slot in a forward phase whose fields are not read afterwards (the
// plan's fused flag) keeps a pitched copy of its state for the fused
// one-launch step from its first such chunk until it leaves the phase.
#pragma once

#include "../../include/tide_b200_serve.h"

#include <cstddef>
#include <map>
#include <tuple>

namespace tb {
namespace {

constexpr int kSrvMaxSlots = 256;
enum SrvKind : int { kSrvFH = 0, kSrvFE = 1, kSrvAE = 2, kSrvAH = 3 };

struct SrvSlot {
  TMGeom<float> g;
  const float *ca, *cb, *cq;
  float *ey, *hx, *hz, *m_ey_x, *m_ey_z, *m_hx_z, *m_hz_x;
  const float *f;
  float *r;
  PointCSR src_e, rec_e, src_ah, rec_ah;
  const unsigned char *rowf_ah;
  float *lam_ey, *lam_hx, *lam_hz;
  float *mem[4][2];  // adjoint memories Ey-x, Ey-z, Hx-z, Hz-x: [caller's, scratch]
  const float *grad_r;
  float *grad_f, *grad_ca, *grad_cb;
  void *ey_st, *cu_st;  // snapshot bases (store index q0 first)
  int64_t shot_cells;   // S * ny * nx
  int64_t fs, rs;       // S * n_src, S * n_rec
  int phase, t0, n, parity, k, q0;
  int gx[4], gy[4];     // tile grid of each kernel kind (z: shots, or 1 for adjoint H)
};

struct SrvTable {
  int n_slots;
  int total[4];
  int pre[4][kSrvMaxSlots + 1];
  SrvSlot slot[kSrvMaxSlots];
};

// Slot of virtual tile vb: pre is an exclusive scan with pre[n] = total.  CTAs
// walk vb upwards, so the search resumes from the previous slot.
__device__ __forceinline__ int srv_find(const int *__restrict__ pre, int n, int vb, int hint) {
  int i = hint;
  if (i < 0) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(pre + mid) <= vb) lo = mid;
      else hi = mid - 1;
    }
    i = lo;
  }
  while (vb >= __ldg(pre + i + 1)) ++i;
  return i;
}

__device__ __forceinline__ Tile srv_tile(const SrvSlot &sl, int kind, int local) {
  const int gx = sl.gx[kind], gy = sl.gy[kind], per = gx * gy;
  return Tile{local % gx, (local % per) / gx, local / per, gx, gy};
}

template <int KIND, typename Body>
__device__ __forceinline__ void srv_walk(const SrvTable *__restrict__ tab, int j, Body body) {
  const int total = tab->total[KIND], n = tab->n_slots;
  int i = -1;
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    i = srv_find(tab->pre[KIND], n, vb, i);
    const SrvSlot &sl = tab->slot[i];
    if (j >= sl.n) continue;  // this slot has run its steps of the chunk
    body(sl, srv_tile(sl, KIND, vb - tab->pre[KIND][i]));
  }
}

__global__ void __launch_bounds__(256, 6) k_srv_fwd_h(const SrvTable *__restrict__ tab, int j) {
  srv_walk<kSrvFH>(tab, j, [&](const SrvSlot &sl, const Tile &tl) {
    const TMGeom<float> &g = sl.g;
    fwd_h_tile<float, kRowsH>(tl, g, sl.cq, sl.ey, sl.hx, sl.hz, sl.m_ey_x, sl.m_ey_z);
  });
}

// Snapshot element type S is fixed per engine (float or bf16), so each kernel
// carries one instantiation of the tile function.
template <typename S>
__global__ void __launch_bounds__(256, 3) k_srv_fwd_e(const SrvTable *__restrict__ tab, int j) {
  srv_walk<kSrvFE>(tab, j, [&](const SrvSlot &sl, const Tile &tl) {
    const TMGeom<float> &g = sl.g;
    const int t = sl.t0 + j;
    const float *f_t = sl.f ? sl.f + (int64_t)t * sl.fs : nullptr;
    float *r_t = sl.r ? sl.r + (int64_t)t * sl.rs : nullptr;
    const bool store = sl.phase == TIDE_SERVE_FORWARD_STORE && t % sl.k == 0;
    const int64_t off = store ? (int64_t)(t / sl.k - sl.q0) * sl.shot_cells : 0;
    S *es = store && sl.ey_st ? static_cast<S *>(sl.ey_st) + off : nullptr;
    S *cs = store && sl.cu_st ? static_cast<S *>(sl.cu_st) + off : nullptr;
    fwd_e_tile<float, S, kRowsE>(tl, g, sl.ca, sl.cb, sl.hx, sl.hz, sl.ey, sl.m_hx_z, sl.m_hz_x,
                                 es, cs, sl.src_e, sl.rec_e, f_t, r_t);
  });
}

__global__ void __launch_bounds__(256, 3) k_srv_adj_e(const SrvTable *__restrict__ tab, int j) {
  srv_walk<kSrvAE>(tab, j, [&](const SrvSlot &sl, const Tile &tl) {
    const TMGeom<float> &g = sl.g;
    const int c = (sl.parity + j) & 1;
    adj_e_tile<float, kRowsAE>(tl, g, sl.cb, sl.lam_ey, sl.lam_hx, sl.lam_hz, sl.mem[2][c],
                               sl.mem[3][c], sl.mem[2][c ^ 1], sl.mem[3][c ^ 1]);
  });
}

template <typename S>
__global__ void __launch_bounds__(256, 3) k_srv_adj_h(const SrvTable *__restrict__ tab, int j) {
  srv_walk<kSrvAH>(tab, j, [&](const SrvSlot &sl, const Tile &tl) {
    const TMGeom<float> &g = sl.g;
    const int c = (sl.parity + j) & 1;
    const int t = sl.t0 - 1 - j;
    const bool img = (sl.ey_st || sl.cu_st) && t % sl.k == 0;
    const int64_t off = img ? (int64_t)(t / sl.k - sl.q0) * sl.shot_cells : 0;
    const float *grt = sl.grad_r ? sl.grad_r + (int64_t)t * sl.rs : nullptr;
    float *gft = sl.grad_f ? sl.grad_f + (int64_t)t * sl.fs : nullptr;
    const S *es = img && sl.ey_st ? static_cast<const S *>(sl.ey_st) + off : nullptr;
    const S *cs = img && sl.cu_st ? static_cast<const S *>(sl.cu_st) + off : nullptr;
    const GradArgs<float, S> ga{es, cs, sl.grad_ca, sl.grad_cb, (float)sl.k, false, false};
    adj_h_tile<float, S, kRowsAH>(tl, g, sl.ca, sl.cq, sl.lam_hx, sl.lam_hz, sl.lam_ey,
                                  sl.mem[0][c], sl.mem[1][c], sl.mem[0][c ^ 1], sl.mem[1][c ^ 1],
                                  sl.rec_ah, sl.src_ah, sl.rowf_ah, grt, gft, ga);
  });
}

// Host side -----------------------------------------------------------------

constexpr int kSrvPool = 8;  // streams of the large slots

struct SrvHostSlot {
  bool bound = false;
  SrvSlot s{};          // static part filled at bind; plan fills the rest
  void *points = nullptr;
  int tiles[4] = {0, 0, 0, 0};  // tiles of each kind
  bool adjoint = false;
  int64_t nt = 0;
  // large slots
  bool direct = false;
  int pool = 0;
  Launch<float, 2> L{};
  bool fused_ok = false;           // plan: fields not read after this forward phase
  PitchedFwd *pf = nullptr;        // pitched state of the fused forward
  PointScratch *pf_pts = nullptr;  // tile lists of the fused tiling
  const int64_t *src_i = nullptr, *rec_i = nullptr;
  int64_t n_src = 0, n_rec = 0;
};

struct SrvEngine {
  int device = 0;
  int max_slots = 0;
  int fmt = 0;  // snapshot format of every job: 0 float32, 1 bf16
  cudaStream_t sf = nullptr, sa = nullptr;
  cudaEvent_t ev_in = nullptr, ev_fork = nullptr, ev_join = nullptr, ev_up[2] = {nullptr, nullptr};
  bool up_pending[2] = {false, false};
  SrvTable *d_table = nullptr;
  SrvTable *h_table[2] = {nullptr, nullptr};
  int cur = 0;
  int grid[4] = {0, 0, 0, 0};
  int64_t direct_cells = (int64_t)1 << 20;  // shots x cells of a large slot (< 0: none)
  bool fused = true;                        // fused forward step for eligible large slots
  int n_pool = kSrvPool;  // streams the large slots are spread over (serve_set_direct_streams)
  cudaStream_t pool[kSrvPool] = {};
  cudaEvent_t ev_pool[kSrvPool] = {};
  std::vector<SrvHostSlot> slots;
  std::map<std::tuple<int, bool, bool>, cudaGraphExec_t> graphs;
  std::vector<std::pair<void *, cudaEvent_t>> deferred;  // released tile lists, freed when done
  int64_t launches = 0;

  // Free the released tile lists whose last reader has finished.
  void sweep(bool wait) {
    size_t keep = 0;
    for (auto &d : deferred) {
      if (wait) cudaEventSynchronize(d.second);
      if (cudaEventQuery(d.second) == cudaSuccess) {
        cudaFree(d.first);
        cudaEventDestroy(d.second);
      } else {
        deferred[keep++] = d;
      }
    }
    deferred.resize(keep);
  }

  ~SrvEngine() {
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    if (sf) cudaStreamSynchronize(sf);
    if (sa) cudaStreamSynchronize(sa);
    sweep(true);
    for (auto &s : slots) {
      delete s.pf;
      delete s.pf_pts;
      if (s.points) cudaFree(s.points);
    }
    for (int i = 0; i < kSrvPool; ++i) {
      if (pool[i]) cudaStreamSynchronize(pool[i]);
      if (ev_pool[i]) cudaEventDestroy(ev_pool[i]);
      if (pool[i]) cudaStreamDestroy(pool[i]);
    }
    if (d_table) cudaFree(d_table);
    for (auto *h : h_table)
      if (h) cudaFreeHost(h);
    for (cudaEvent_t e : {ev_in, ev_fork, ev_join, ev_up[0], ev_up[1]})
      if (e) cudaEventDestroy(e);
    if (sf) cudaStreamDestroy(sf);
    if (sa) cudaStreamDestroy(sa);
  }
};

// Launches of one chunk: forward chain on sf, adjoint chain on sa.
void srv_enqueue(SrvEngine &E, int C, bool fwd, bool adj) {
  const dim3 block(kTileX, kBlockY, 1);
  if (TB_CUDA(cudaEventRecord(E.ev_fork, E.sf))) return;
  if (TB_CUDA(cudaStreamWaitEvent(E.sa, E.ev_fork, 0))) return;
  using B = __nv_bfloat16;
  for (int j = 0; j < C; ++j) {
    if (fwd) {
      k_srv_fwd_h<<<E.grid[kSrvFH], block, 0, E.sf>>>(E.d_table, j);
      if (E.fmt) k_srv_fwd_e<B><<<E.grid[kSrvFE], block, 0, E.sf>>>(E.d_table, j);
      else k_srv_fwd_e<float><<<E.grid[kSrvFE], block, 0, E.sf>>>(E.d_table, j);
    }
    if (adj) {
      k_srv_adj_e<<<E.grid[kSrvAE], block, 0, E.sa>>>(E.d_table, j);
      if (E.fmt) k_srv_adj_h<B><<<E.grid[kSrvAH], block, 0, E.sa>>>(E.d_table, j);
      else k_srv_adj_h<float><<<E.grid[kSrvAH], block, 0, E.sa>>>(E.d_table, j);
    }
  }
  if (TB_CUDA(cudaEventRecord(E.ev_join, E.sa))) return;
  TB_CUDA(cudaStreamWaitEvent(E.sf, E.ev_join, 0));
}

// Steps of one large slot with the per-call kernels on stream st.
template <typename S>
bool srv_direct(SrvHostSlot &H, cudaStream_t st, bool fused_enabled, int64_t &launches) {
  SrvSlot &s = H.s;
  const Launch<float, 2> &L = H.L;
  PointScratch pe, pa;  // views of the slot's lists (own no memory)
  pe.src = s.src_e; pe.rec = s.rec_e;
  pa.src = s.src_ah; pa.rec = s.rec_ah; pa.rowf = s.rowf_ah;
  const bool fwd = s.phase == TIDE_SERVE_FORWARD || s.phase == TIDE_SERVE_FORWARD_STORE;
  bool fused = fwd && H.fused_ok && fused_enabled && fused_pays(s.g.n_shots, s.g.N);
  if (fused && !H.pf) {
    // entering the fused phase needs a pitched copy of the slot's state; when
    // the free device memory cannot take it (the caller's allocator may hold
    // the rest) the slot runs the per-call pair, which gives the same bits
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess ||
        free_b < PitchedFwd::bytes_for(s.g) + ((size_t)1 << 30)) {
      cudaGetLastError();
      fused = false;
    }
  }
  if (H.pf && !fused) {
    // leaving the fused phase: fields back to the caller's layout when a
    // forward follows, then the pitched copy goes
    if (fwd && !H.pf->finish()) return false;
    delete H.pf;
    delete H.pf_pts;
    H.pf = nullptr;
    H.pf_pts = nullptr;
  }
  if (fused && !H.pf) {
    H.pf = new PitchedFwd();
    float *const fields[7] = {s.ey, s.hx, s.hz, s.m_ey_x, s.m_ey_z, s.m_hx_z, s.m_hz_x};
    if (!H.pf->init(L.g, fields, s.ca, s.cb, s.cq, st)) return false;
    H.pf_pts = new PointScratch();
    if (!build_points(*H.pf_pts, L, H.pf->q.pt, H.src_i, H.n_src, H.rec_i, H.n_rec, st))
      return false;
  }
  const DebyeArgs<float> db{nullptr, nullptr, nullptr, nullptr, 0};
  for (int j = 0; j < s.n; ++j) {
    if (fwd) {
      const int64_t t = s.t0 + j;
      const float *ft = s.f ? s.f + t * s.fs : nullptr;
      float *rt = s.r ? s.r + t * s.rs : nullptr;
      const bool store = s.phase == TIDE_SERVE_FORWARD_STORE && t % s.k == 0;
      const int64_t off = store ? (t / s.k - s.q0) * s.shot_cells : 0;
      S *es = store && s.ey_st ? static_cast<S *>(s.ey_st) + off : nullptr;
      S *cs = store && s.cu_st ? static_cast<S *>(s.cu_st) + off : nullptr;
      if (fused) {
        H.pf->launch<S>(L.g, es, cs, *H.pf_pts, ft, rt);
        launches += 1;
      } else {
        launch_fwd_h<float, 2>(L, st, s.cq, s.ey, s.hx, s.hz, s.m_ey_x, s.m_ey_z);
        launch_fwd_e<float, 2, S>(L, st, s.ca, s.cb, s.hx, s.hz, s.ey, s.m_hx_z, s.m_hz_x, es,
                                  cs, db, pe, ft, rt);
        launches += 2;
      }
    } else {
      const int64_t t = s.t0 - 1 - j;
      const int c = (s.parity + j) & 1;
      launch_adj_e<float, 2>(L, st, s.cb, s.lam_ey, s.lam_hx, s.lam_hz, s.mem[2][c], s.mem[3][c],
                             s.mem[2][c ^ 1], s.mem[3][c ^ 1]);
      const bool img = (s.ey_st || s.cu_st) && t % s.k == 0;
      const int64_t off = img ? (t / s.k - s.q0) * s.shot_cells : 0;
      const S *es = img && s.ey_st ? static_cast<const S *>(s.ey_st) + off : nullptr;
      const S *cs = img && s.cu_st ? static_cast<const S *>(s.cu_st) + off : nullptr;
      const GradArgs<float, S> ga{es, cs, s.grad_ca, s.grad_cb, (float)s.k, false, false};
      launch_adj_h<float, 2, S>(L, st, s.ca, s.cq, s.lam_hx, s.lam_hz, s.lam_ey, s.mem[0][c],
                                s.mem[1][c], s.mem[0][c ^ 1], s.mem[1][c ^ 1], pa,
                                s.grad_r ? s.grad_r + t * s.rs : nullptr,
                                s.grad_f ? s.grad_f + t * s.fs : nullptr, ga);
      launches += 2;
    }
  }
  return true;
}

bool srv_points(const int64_t *idx, int64_t n_per_shot, int64_t S, int64_t N, int nx,
                const PointTiles &pt, int *&w, cudaStream_t st, PointCSR &out) {
  out = PointCSR{nullptr, nullptr, nullptr};
  if (n_per_shot <= 0 || idx == nullptr) return true;
  const int n_tiles = pt.tiles_x * pt.tiles_y * (int)S;
  const size_t nt1 = (size_t)n_tiles + 1, n = (size_t)(n_per_shot * S);
  int *count = w, *start = w + nt1, *cell = w + 2 * nt1, *ent = w + 2 * nt1 + n;
  w += 2 * nt1 + 2 * n;
  return build_list(idx, (int)n_per_shot, (int)S, N, nx, pt, n_tiles, count, start, cell, ent,
                    st, out);
}

}  // namespace
}  // namespace tb

extern "C" {

void *tide_b200_serve_create(int64_t device, int64_t max_slots, int64_t storage_format) {
  using namespace tb;
  if (max_slots < 1 || max_slots > kSrvMaxSlots) {
    set_error(kBadArgument, "serve: max_slots must be in [1, %d]", kSrvMaxSlots);
    return nullptr;
  }
  if (storage_format != 0 && storage_format != 1) {
    set_error(kBadArgument, "serve: storage_format must be 0 (float32) or 1 (bf16)");
    return nullptr;
  }
  if (TB_CUDA(cudaSetDevice((int)device))) return nullptr;
  auto *E = new SrvEngine();
  E->device = (int)device;
  E->max_slots = (int)max_slots;
  E->fmt = (int)storage_format;
  E->slots.resize((size_t)max_slots);
  bool ok = !TB_CUDA(cudaStreamCreateWithFlags(&E->sf, cudaStreamNonBlocking)) &&
            !TB_CUDA(cudaStreamCreateWithFlags(&E->sa, cudaStreamNonBlocking));
  for (cudaEvent_t *e : {&E->ev_in, &E->ev_fork, &E->ev_join, &E->ev_up[0], &E->ev_up[1]})
    ok = ok && !TB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  for (int i = 0; ok && i < kSrvPool; ++i)
    ok = !TB_CUDA(cudaStreamCreateWithFlags(&E->pool[i], cudaStreamNonBlocking)) &&
         !TB_CUDA(cudaEventCreateWithFlags(&E->ev_pool[i], cudaEventDisableTiming));
  ok = ok && !TB_CUDA(cudaMalloc(&E->d_table, sizeof(SrvTable)));
  for (auto *&h : E->h_table)
    ok = ok && !TB_CUDA(cudaMallocHost(&h, sizeof(SrvTable)));
  int sms = 0;
  ok = ok && !TB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, (int)device));
  using B = __nv_bfloat16;
  const void *kern[4] = {
      (const void *)k_srv_fwd_h,
      E->fmt ? (const void *)k_srv_fwd_e<B> : (const void *)k_srv_fwd_e<float>,
      (const void *)k_srv_adj_e,
      E->fmt ? (const void *)k_srv_adj_h<B> : (const void *)k_srv_adj_h<float>};
  for (int k = 0; ok && k < 4; ++k) {
    int per = 0;
    ok = !TB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern[k], kTileX * kBlockY, 0));
    E->grid[k] = sms * std::max(per, 1);
  }
  if (!ok) {
    delete E;
    return nullptr;
  }
  return E;
}

void tide_b200_serve_destroy(void *engine) {
  auto *E = static_cast<tb::SrvEngine *>(engine);
  if (E == nullptr) return;
  cudaSetDevice(E->device);
  delete E;
}

int64_t tide_b200_serve_bind(void *engine, const TideServeJob *job, int64_t stream) {
  using namespace tb;
  auto *E = static_cast<SrvEngine *>(engine);
  if (E == nullptr || job == nullptr) {
    set_error(kBadArgument, "serve bind: null engine or job");
    return -1;
  }
  if (TB_CUDA(cudaSetDevice(E->device))) return -1;
  const TideServeJob &J = *job;
  if (J.ny < 3 || J.nx < 3 || J.n_shots < 1 || J.nt < 0 || J.n_src < 0 || J.n_rec < 0 ||
      J.ny * J.nx > ((int64_t)1 << 31) - 1 || J.n_shots > 65535) {
    set_error(kBadArgument, "serve bind: unsupported shape S=%lld ny=%lld nx=%lld nt=%lld",
              (long long)J.n_shots, (long long)J.ny, (long long)J.nx, (long long)J.nt);
    return -1;
  }
  if (!J.ca || !J.cb || !J.cq || !J.ey || !J.hx || !J.hz || !J.m_ey_x || !J.m_ey_z ||
      !J.m_hx_z || !J.m_hz_x || (J.n_src > 0 && (!J.f || !J.sources_i)) ||
      (J.n_rec > 0 && (!J.r || !J.receivers_i))) {
    set_error(kBadArgument, "serve bind: a required buffer is null");
    return -1;
  }
  const bool adjoint = J.lam[0] != nullptr;
  if (adjoint) {
    for (int k = 0; k < 7; ++k)
      if (!J.lam[k]) {
        set_error(kBadArgument, "serve bind: adjoint buffer %d is null", k);
        return -1;
      }
    if (!J.lam_scratch || (J.n_rec > 0 && !J.grad_r) || J.step_ratio < 1 ||
        J.storage_format != E->fmt) {
      set_error(kBadArgument, "serve bind: bad adjoint arguments");
      return -1;
    }
  }
  int slot = -1;
  for (int i = 0; i < E->max_slots; ++i)
    if (!E->slots[(size_t)i].bound) {
      slot = i;
      break;
    }
  if (slot < 0) {
    set_error(kBadArgument, "serve bind: all %d slots are in use", E->max_slots);
    return -1;
  }
  Launch<float, 2> L;
  if (!make_launch(L, J.ay, J.by, J.ayh, J.byh, J.ax, J.bx, J.axh, J.bxh, J.ky, J.kyh, J.kx,
                   J.kxh, (float)J.rdy, (float)J.rdx, J.n_shots, J.ny, J.nx, J.pml_y0, J.pml_x0,
                   J.pml_y1, J.pml_x1, false, false, false))
    return -1;
  SrvHostSlot &H = E->slots[(size_t)slot];
  H = SrvHostSlot{};
  SrvSlot &s = H.s;
  s.g = L.g;
  s.ca = J.ca; s.cb = J.cb; s.cq = J.cq;
  s.ey = J.ey; s.hx = J.hx; s.hz = J.hz;
  s.m_ey_x = J.m_ey_x; s.m_ey_z = J.m_ey_z; s.m_hx_z = J.m_hx_z; s.m_hz_x = J.m_hz_x;
  s.f = J.n_src > 0 ? J.f : nullptr;
  s.r = J.n_rec > 0 ? J.r : nullptr;
  s.shot_cells = J.n_shots * J.ny * J.nx;
  s.fs = J.n_shots * J.n_src;
  s.rs = J.n_shots * J.n_rec;
  s.k = (int)std::max<int64_t>(1, J.step_ratio);
  const int S = (int)J.n_shots;
  const int gx[4] = {(int)L.grid_h.x, (int)L.grid_e.x, (int)L.grid_ae.x, (int)L.grid_ah.x};
  const int gy[4] = {(int)L.grid_h.y, (int)L.grid_e.y, (int)L.grid_ae.y, (int)L.grid_ah.y};
  const int gz[4] = {S, S, S, 1};
  for (int k = 0; k < 4; ++k) {
    s.gx[k] = gx[k];
    s.gy[k] = gy[k];
    H.tiles[k] = gx[k] * gy[k] * gz[k];
  }
  H.adjoint = adjoint;
  H.nt = J.nt;
  H.direct = E->direct_cells >= 0 && s.shot_cells >= E->direct_cells;
  H.pool = slot % E->n_pool;
  H.L = L;
  if (H.direct) H.L.narrow_e();  // the per-call E kernels' block shape
  H.src_i = J.n_src > 0 ? J.sources_i : nullptr;
  H.rec_i = J.n_rec > 0 ? J.receivers_i : nullptr;
  H.n_src = J.n_src;
  H.n_rec = J.n_rec;
  if (adjoint) {
    s.lam_ey = J.lam[0]; s.lam_hx = J.lam[1]; s.lam_hz = J.lam[2];
    const size_t SN = (size_t)s.shot_cells;
    for (int m = 0; m < 4; ++m) {
      s.mem[m][0] = J.lam[3 + m];
      s.mem[m][1] = J.lam_scratch + m * SN;
    }
    s.grad_r = J.n_rec > 0 ? J.grad_r : nullptr;
    s.grad_f = J.n_src > 0 ? J.grad_f : nullptr;
    s.grad_ca = J.grad_ca;
    s.grad_cb = J.grad_cb;
  }
  // Tile lists: E tiling (forward; the table walk's, or for a large slot that
  // of the per-call E kernel) and, for the adjoint, adjoint-H tiling.
  const PointTiles pe = H.direct ? H.L.e_tiles()
                                 : PointTiles{L.tiles_x, L.tiles_y_e, kTileX, kBlockY * kRowsE, 0};
  const PointTiles ph = L.ah_tiles();  // 8-warp blocks: the table's tiling
  auto words = [&](const PointTiles &pt, int64_t per) -> size_t {
    if (per <= 0) return 0;
    return 2 * ((size_t)pt.tiles_x * pt.tiles_y * S + 1) + 2 * (size_t)(per * S);
  };
  size_t w = words(pe, J.n_src) + words(pe, J.n_rec);
  if (adjoint) w += words(ph, J.n_src) + words(ph, J.n_rec);
  const size_t n_rows = adjoint ? (size_t)L.tiles_y_ah * S : 0;
  cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  if (TB_CUDA(cudaEventRecord(E->ev_in, caller))) return -1;
  if (TB_CUDA(cudaStreamWaitEvent(E->sf, E->ev_in, 0))) return -1;
  auto fail = [&]() -> int64_t {
    if (H.points) {
      cudaStreamSynchronize(E->sf);
      cudaFree(H.points);
    }
    H = SrvHostSlot{};
    return -1;
  };
  if (w + n_rows > 0) {
    if (TB_CUDA(cudaMalloc(&H.points, w * sizeof(int) + n_rows + 16))) return fail();
    int *p = static_cast<int *>(H.points);
    const int N = (int)(J.ny * J.nx);
    if (!srv_points(J.sources_i, J.n_src, S, N, (int)J.nx, pe, p, E->sf, s.src_e) ||
        !srv_points(J.receivers_i, J.n_rec, S, N, (int)J.nx, pe, p, E->sf, s.rec_e))
      return fail();
    if (adjoint) {
      if (!srv_points(J.sources_i, J.n_src, S, N, (int)J.nx, ph, p, E->sf, s.src_ah) ||
          !srv_points(J.receivers_i, J.n_rec, S, N, (int)J.nx, ph, p, E->sf, s.rec_ah))
        return fail();
      auto *rowf = reinterpret_cast<unsigned char *>(p);
      k_points_rowflags<<<(unsigned)((n_rows + 255) / 256), 256, 0, E->sf>>>(
          s.src_ah.start, s.rec_ah.start, L.tiles_x, (int)n_rows, rowf);
      count_launches(1);
      s.rowf_ah = rowf;
    }
  }
  if (TB_CUDA(cudaGetLastError())) return fail();
  s.phase = TIDE_SERVE_IDLE;
  H.bound = true;
  return slot;
}

int64_t tide_b200_serve_release(void *engine, int64_t slot) {
  using namespace tb;
  auto *E = static_cast<SrvEngine *>(engine);
  if (E == nullptr || slot < 0 || slot >= E->max_slots || !E->slots[(size_t)slot].bound) {
    set_error(kBadArgument, "serve release: bad slot %lld", (long long)slot);
    return -1;
  }
  if (TB_CUDA(cudaSetDevice(E->device))) return -1;
  SrvHostSlot &H = E->slots[(size_t)slot];
  delete H.pf;      // stream-ordered frees on the slot's pool stream
  delete H.pf_pts;
  if (H.points) {
    // enqueued chunks may still read the slot's tile lists: free them once
    // the engine's stream has passed this point
    cudaEvent_t ev = nullptr;
    if (TB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming))) return -1;
    if (TB_CUDA(cudaEventRecord(ev, E->sf))) {
      cudaEventDestroy(ev);
      return -1;
    }
    E->deferred.emplace_back(H.points, ev);
  }
  H = SrvHostSlot{};
  E->sweep(false);
  return 0;
}

int64_t tide_b200_serve_plan(void *engine, int64_t slot, int64_t phase, int64_t t0,
                             int64_t n_steps, void *ey_store, void *curl_store, int64_t q0,
                             int64_t adj_parity, int64_t flags) {
  using namespace tb;
  auto *E = static_cast<SrvEngine *>(engine);
  if (E == nullptr || slot < 0 || slot >= E->max_slots || !E->slots[(size_t)slot].bound) {
    set_error(kBadArgument, "serve plan: bad slot %lld", (long long)slot);
    return -1;
  }
  SrvHostSlot &H = E->slots[(size_t)slot];
  SrvSlot &s = H.s;
  const bool fwd = phase == TIDE_SERVE_FORWARD || phase == TIDE_SERVE_FORWARD_STORE;
  if (phase < TIDE_SERVE_IDLE || phase > TIDE_SERVE_ADJOINT || n_steps < 0 || t0 < 0 ||
      (fwd && t0 + n_steps > H.nt) ||
      (phase == TIDE_SERVE_ADJOINT && (!H.adjoint || t0 > H.nt || t0 - n_steps < 0))) {
    set_error(kBadArgument, "serve plan: bad phase/t0/n_steps (%lld, %lld, %lld)",
              (long long)phase, (long long)t0, (long long)n_steps);
    return -1;
  }
  if (phase == TIDE_SERVE_FORWARD_STORE && !ey_store && !curl_store) {
    set_error(kBadArgument, "serve plan: forward-with-storage needs a snapshot buffer");
    return -1;
  }
  s.phase = (int)phase;
  s.t0 = (int)t0;
  s.n = (int)n_steps;
  s.ey_st = (phase == TIDE_SERVE_FORWARD_STORE || phase == TIDE_SERVE_ADJOINT) ? ey_store : nullptr;
  s.cu_st = (phase == TIDE_SERVE_FORWARD_STORE || phase == TIDE_SERVE_ADJOINT) ? curl_store : nullptr;
  s.q0 = (int)q0;
  s.parity = (int)(adj_parity & 1);
  H.fused_ok = (flags & TIDE_SERVE_FLAG_FUSED) != 0;
  return 0;
}

int64_t tide_b200_serve_run(void *engine, int64_t chunk_steps, int64_t use_graph,
                            int64_t stream) {
  using namespace tb;
  auto *E = static_cast<SrvEngine *>(engine);
  if (E == nullptr || chunk_steps < 1 || chunk_steps > 4096) {
    set_error(kBadArgument, "serve run: bad engine or chunk_steps");
    return -1;
  }
  if (TB_CUDA(cudaSetDevice(E->device))) return -1;
  const int C = (int)chunk_steps;
  // Work table of this chunk in the pinned buffer not read by a pending copy.
  const int b = E->cur;
  if (E->up_pending[b] && TB_CUDA(cudaEventSynchronize(E->ev_up[b]))) return -1;
  SrvTable &T = *E->h_table[b];
  int n = 0;
  bool any_f = false, any_a = false;
  for (int k = 0; k < 4; ++k) T.pre[k][0] = 0;
  bool any_direct = false;
  for (auto &H : E->slots) {
    if (!H.bound || H.s.phase == TIDE_SERVE_IDLE || H.s.n <= 0) continue;
    if (H.direct) {
      any_direct = true;
      continue;
    }
    const bool adj = H.s.phase == TIDE_SERVE_ADJOINT;
    any_f = any_f || !adj;
    any_a = any_a || adj;
    T.slot[n] = H.s;
    for (int k = 0; k < 4; ++k) {
      const bool on = (k >= kSrvAE) == adj;
      T.pre[k][n + 1] = T.pre[k][n] + (on ? H.tiles[k] : 0);
    }
    ++n;
  }
  T.n_slots = n;
  for (int k = 0; k < 4; ++k) T.total[k] = T.pre[k][n];
  if (n == 0 && !any_direct) return 0;
  cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  if (TB_CUDA(cudaEventRecord(E->ev_in, caller))) return -1;
  if (TB_CUDA(cudaStreamWaitEvent(E->sf, E->ev_in, 0))) return -1;
  // large slots: per-call kernels on the pool streams, after the caller's work
  bool used[kSrvPool] = {};
  int64_t nl_direct = 0;
  for (auto &H : E->slots) {
    if (!H.bound || !H.direct || H.s.phase == TIDE_SERVE_IDLE || H.s.n <= 0) continue;
    cudaStream_t ps = E->pool[H.pool];
    if (!used[H.pool]) {
      if (TB_CUDA(cudaStreamWaitEvent(ps, E->ev_in, 0))) return -1;
      used[H.pool] = true;
    }
    const bool ok = E->fmt ? srv_direct<__nv_bfloat16>(H, ps, E->fused, nl_direct)
                           : srv_direct<float>(H, ps, E->fused, nl_direct);
    if (!ok) return -1;
  }
  for (auto &H : E->slots)  // steps are consumed: a slot runs again only when re-planned
    if (H.bound) H.s.n = 0;
  auto join_pool = [&]() -> bool {
    for (int i = 0; i < kSrvPool; ++i)
      if (used[i] && (TB_CUDA(cudaEventRecord(E->ev_pool[i], E->pool[i])) ||
                      TB_CUDA(cudaStreamWaitEvent(E->sf, E->ev_pool[i], 0))))
        return false;
    return true;
  };
  E->launches += nl_direct;
  count_launches(nl_direct);
  if (n == 0) {
    if (!join_pool()) return -1;
    if (TB_CUDA(cudaEventRecord(E->ev_in, E->sf))) return -1;
    if (TB_CUDA(cudaStreamWaitEvent(caller, E->ev_in, 0))) return -1;
    return TB_CUDA(cudaGetLastError()) ? -1 : 0;
  }
  const size_t bytes = offsetof(SrvTable, slot) + (size_t)n * sizeof(SrvSlot);
  if (TB_CUDA(cudaMemcpyAsync(E->d_table, &T, bytes, cudaMemcpyHostToDevice, E->sf))) return -1;
  if (TB_CUDA(cudaEventRecord(E->ev_up[b], E->sf))) return -1;
  E->up_pending[b] = true;
  E->cur ^= 1;
  const int64_t nl = (int64_t)C * (2 * (int)any_f + 2 * (int)any_a);
  if (use_graph) {
    const auto key = std::make_tuple(C, any_f, any_a);
    auto it = E->graphs.find(key);
    if (it == E->graphs.end()) {
      cudaGraph_t g = nullptr;
      cudaGraphExec_t ge = nullptr;
      if (TB_CUDA(cudaStreamBeginCapture(E->sf, cudaStreamCaptureModeThreadLocal))) return -1;
      srv_enqueue(*E, C, any_f, any_a);
      const bool bad = TB_CUDA(cudaStreamEndCapture(E->sf, &g));
      if (bad || TB_CUDA(cudaGraphInstantiate(&ge, g, 0))) {
        if (g) cudaGraphDestroy(g);
        return -1;
      }
      cudaGraphDestroy(g);
      it = E->graphs.emplace(key, ge).first;
    }
    if (TB_CUDA(cudaGraphLaunch(it->second, E->sf))) return -1;
  } else {
    srv_enqueue(*E, C, any_f, any_a);
  }
  E->launches += nl;
  count_launches(nl);
  if (!join_pool()) return -1;
  if (TB_CUDA(cudaGetLastError())) return -1;
  if (TB_CUDA(cudaEventRecord(E->ev_in, E->sf))) return -1;
  if (TB_CUDA(cudaStreamWaitEvent(caller, E->ev_in, 0))) return -1;
  return 0;
}

int64_t tide_b200_serve_configure(void *engine, int64_t direct_cells, int64_t fused) {
  auto *E = static_cast<tb::SrvEngine *>(engine);
  if (E == nullptr) {
    tb::set_error(tb::kBadArgument, "serve configure: null engine");
    return -1;
  }
  E->direct_cells = direct_cells;
  E->fused = fused != 0;
  return 0;
}

int64_t tide_b200_serve_set_direct_streams(void *engine, int64_t n) {
  auto *E = static_cast<tb::SrvEngine *>(engine);
  if (E == nullptr || n < 1 || n > tb::kSrvPool) {
    tb::set_error(tb::kBadArgument, "serve set_direct_streams: null engine or n outside [1, %d]",
                  tb::kSrvPool);
    return -1;
  }
  const int prev = E->n_pool;
  E->n_pool = (int)n;
  return prev;
}

int64_t tide_b200_serve_launches(void *engine) {
  auto *E = static_cast<tb::SrvEngine *>(engine);
  return E ? E->launches : -1;
}

}  // extern "C"
