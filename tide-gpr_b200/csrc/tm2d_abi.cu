// extern "C" entry points of the TM2D path: forward, forward_with_storage and
// backward for stencil orders 2/4/6/8 in float and double, under the
// reference's symbol names (see include/tide_b200.h for the interface each
// one replaces).  The serving engine (tm2d_serve.cuh), the Debye gradient
// (tm2d_debye.cuh) and the Born passes (tm2d_born.cuh) are compiled into this
// translation unit from the includes at its end; the snapshot pipeline of the
// storing forwards is StoreRun (tb_store.cuh).
//
// Every call works on the caller's stream (compute_stream; 0 = legacy
// default) and returns as soon as its work is enqueued, except that the cpu
// and disk storage modes synchronise their copies before returning, as the
// reference does (maxwell_tm_cuda_inst.cu:1601-1604); the disk mode also
// waits for its file writes.
#include <algorithm>
#include <atomic>
#include <memory>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "../../include/tide_b200.h"
#include "tb_common.cuh"
#include "tm2d_kernels.cuh"
#include "tm2d_fused.cuh"
#include "tm2d_s2.cuh"
#include "tm2d_tma.cuh"
#include "tb_store.cuh"

namespace tb {
namespace {

constexpr int kRing = kStoreRing;  // device ring slots of the cpu / disk storage modes

inline cudaStream_t as_stream(void *h) { return reinterpret_cast<cudaStream_t>(h); }

// Rows per thread of each stencil kernel (see tm2d_kernels.cuh).
constexpr int kRowsH = 1;   // forward H
constexpr int kRowsE = 2;   // forward E (+ storage, points)
constexpr int kRowsAE = 2;  // adjoint E
constexpr int kRowsAH = 1;  // adjoint H (+ points, gradient)

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)std::max<int64_t>(1, (a + b - 1) / b); }

template <typename T, int ST> struct Launch {
  TMGeom<T> g;
  dim3 block{kTileX, kBlockY, 1};
  dim3 grid_h, grid_e, grid_ae, grid_ah;
  int tiles_x = 0, tiles_y_e = 0, tiles_y_ah = 0;
  int ah_by = kBlockY;  // warps per block (rows of 32 cells) of the adjoint H kernel
  // Warps per block of the per-call stencil-2 E and adjoint E kernels
  // (narrow_e); the serving engine and the other kernels keep kBlockY.
  int e_by = kBlockY, ae_by = kBlockY;
  dim3 grid_e_n, grid_ae_n;
  int tiles_y_e_n = 0;
  bool has_domain = false;
  // Point-list tiles of the adjoint H kernel.
  PointTiles ah_tiles() const { return PointTiles{tiles_x, tiles_y_ah, kTileX, ah_by * kRowsAH, 0}; }
  // Point-list tiles of the forward E kernel launch_fwd_e runs.
  PointTiles e_tiles() const {
    return e_by == kBlockY ? PointTiles{tiles_x, tiles_y_e, kTileX, kBlockY * kRowsE, 0}
                           : PointTiles{tiles_x, tiles_y_e_n, kTileX, e_by * kRowsE, 0};
  }
  void set_ah_by(int by) {
    ah_by = by;
    tiles_y_ah = (int)cdiv(g.ny, by * kRowsAH);
    grid_ah = dim3((unsigned)tiles_x, (unsigned)tiles_y_ah, 1);
  }
  // 4-warp blocks for the E and adjoint E kernels of a per-call loop: on the
  // 553 x 1065 grid at 8 shots the stencil-2 forward E kernel runs 34.2
  // against 38.2 us per launch and the adjoint E kernel 26.5 against 28.5;
  // at stencil 4 the generic kernels 44.1 / 65.8 against 45.1 / 69.9, at
  // stencil 8 50.1 / 131 against 51.1 / 135 (the H kernels are faster with
  // 8 warps).  The point lists of a call follow e_tiles(); callers with
  // Debye poles keep the 8-warp forward E launch.
  void narrow_e() {
    constexpr int P = FD<ST>::P;
    e_by = ae_by = kNarrowBY;
    tiles_y_e_n = (int)cdiv(g.ny, kNarrowBY * kRowsE);
    grid_e_n = dim3((unsigned)tiles_x, (unsigned)tiles_y_e_n, (unsigned)g.n_shots);
    grid_ae_n = dim3(cdiv(g.nx - 2 * P + 1, kTileX), cdiv(g.ny - 2 * P + 1, kNarrowBY * kRowsAE),
                     (unsigned)g.n_shots);
  }
  static constexpr int kNarrowBY = 4;
};

template <typename T, int ST>
bool make_launch(Launch<T, ST> &L, const T *ay, const T *by, const T *ayh, const T *byh,
                 const T *ax, const T *bx, const T *axh, const T *bxh, const T *ky,
                 const T *kyh, const T *kx, const T *kxh, T rdy, T rdx, int64_t n_shots,
                 int64_t ny, int64_t nx, int64_t pml_y0, int64_t pml_x0, int64_t pml_y1,
                 int64_t pml_x1, bool ca_b, bool cb_b, bool cq_b) {
  constexpr int P = FD<ST>::P;
  if (n_shots < 1 || n_shots > 65535 || ny < 1 || nx < 1 || ny > (1 << 30) ||
      nx > (1 << 30) || ny * nx > ((int64_t)1 << 31) - 1) {
    set_error(kBadArgument, "TM2D: unsupported shape n_shots=%lld ny=%lld nx=%lld",
              (long long)n_shots, (long long)ny, (long long)nx);
    return false;
  }
  if (!ay || !by || !ayh || !byh || !ax || !bx || !axh || !bxh || !ky || !kyh || !kx || !kxh) {
    set_error(kBadArgument, "TM2D: a CPML profile pointer is null");
    return false;
  }
  TMGeom<T> &g = L.g;
  g.ay = ay; g.by = by; g.ayh = ayh; g.byh = byh;
  g.ax = ax; g.bx = bx; g.axh = axh; g.bxh = bxh;
  g.ky = ky; g.kyh = kyh; g.kx = kx; g.kxh = kxh;
  g.rdy = rdy; g.rdx = rdx;
  g.ny = (int)ny; g.nx = (int)nx; g.N = ny * nx; g.n_shots = (int)n_shots;
  g.pml_y0 = (int)pml_y0; g.pml_y1 = (int)pml_y1;
  g.pml_x0 = (int)pml_x0; g.pml_x1 = (int)pml_x1;
  g.pml_y1h = pml_y1 > pml_y0 ? (int)pml_y1 - 1 : (int)pml_y0;
  g.pml_x1h = pml_x1 > pml_x0 ? (int)pml_x1 - 1 : (int)pml_x0;
  g.ca_b = ca_b; g.cb_b = cb_b; g.cq_b = cq_b;
  const int64_t dx = nx - 2 * P + 1, dy = ny - 2 * P + 1;
  L.has_domain = dx > 0 && dy > 0;
  const unsigned S = (unsigned)n_shots;
  L.grid_h = dim3(cdiv(dx, kTileX), cdiv(dy, kBlockY * kRowsH), S);
  L.grid_ae = dim3(cdiv(dx, kTileX), cdiv(dy, kBlockY * kRowsAE), S);
  L.tiles_x = (int)cdiv(nx, kTileX);
  L.tiles_y_e = (int)cdiv(ny, kBlockY * kRowsE);
  L.grid_e = dim3((unsigned)L.tiles_x, (unsigned)L.tiles_y_e, S);
  L.set_ah_by(kBlockY);
  return true;
}

// Block height of the stencil-2 adjoint H kernel for one call.  Its blocks
// each loop over all shots, so its grid is only a few waves deep (553 x 1065:
// 2380 blocks of 8 warps on 148 x 4 slots = 4.02 waves; 4726 blocks of 4
// warps on 148 x 8 slots = 3.99).  Picks the height whose last wave is
// fullest; on that grid 4 warps run 47.1 us per step against 47.7 at 8 shots.
template <typename T, typename S> void pick_adj_h_rows(Launch<T, 2> &L) {
  static const std::pair<int, int> occ = [] {
    int a = 0, b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k2_adj_h<T, S, kRowsAH, 8>, 256, 0) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k2_adj_h<T, S, kRowsAH, 4>, 128, 0) !=
            cudaSuccess) {
      cudaGetLastError();
      return std::pair<int, int>(0, 0);
    }
    return std::pair<int, int>(a, b);
  }();
  int dev = 0, n_sm = 0;
  if (occ.first < 1 || occ.second < 1 || cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  auto fill = [&](int by, int blocks_per_sm) {
    const double w =
        (double)L.tiles_x * (double)cdiv(L.g.ny, by * kRowsAH) / ((double)n_sm * blocks_per_sm);
    return w / std::ceil(w);
  };
  L.set_ah_by(fill(4, occ.second) > fill(8, occ.first) + 0.02 ? 4 : 8);
}

// Per-call scratch: CSR point lists for sources and receivers, allocated from
// the stream-ordered pool and released at the end of the call.
struct PointScratch {
  void *mem = nullptr;
  cudaStream_t st = nullptr;
  PointCSR src{nullptr, nullptr, nullptr};
  PointCSR rec{nullptr, nullptr, nullptr};
  const unsigned char *rowf = nullptr;  // per (shot, tile row): any point? (null: none at all)
  ~PointScratch() {
    if (mem) cudaFreeAsync(mem, st);
  }
};

bool build_list(const int64_t *idx, int n_per_shot, int n_shots, int64_t N, int nx,
                const PointTiles &pt, int n_tiles, int *count, int *start, int *cell, int *ent,
                cudaStream_t st, PointCSR &out) {
  const int n = n_per_shot * n_shots;
  if (TB_CUDA(cudaMemsetAsync(count, 0, sizeof(int) * n_tiles, st))) return false;
  const int thr = 256, blk = (n + thr - 1) / thr;
  k_points_count<<<blk, thr, 0, st>>>(idx, n_per_shot, n_shots, N, nx, pt, count);
  k_points_scan<<<1, 1024, 0, st>>>(count, start, n_tiles);
  k_points_fill<<<blk, thr, 0, st>>>(idx, n_per_shot, n_shots, N, nx, pt, start, cell, ent);
  if (TB_CUDA(cudaGetLastError())) return false;
  count_launches(3);
  out = PointCSR{start, cell, ent};
  return true;
}

// Point lists for the tiles `pt`.
template <typename T, int ST>
bool build_points(PointScratch &ps, const Launch<T, ST> &L, const PointTiles &pt,
                  const int64_t *sources_i, int64_t n_src, const int64_t *receivers_i,
                  int64_t n_rec, cudaStream_t st) {
  ps.st = st;
  const bool want_s = n_src > 0 && sources_i != nullptr;
  const bool want_r = n_rec > 0 && receivers_i != nullptr;
  if (!want_s && !want_r) return true;
  const int64_t S = L.g.n_shots;
  if ((want_s && n_src * S > (1 << 30)) || (want_r && n_rec * S > (1 << 30))) {
    set_error(kBadArgument, "TM2D: too many source/receiver entries");
    return false;
  }
  const int n_tiles = pt.tiles_x * pt.tiles_y * (int)S;
  const size_t nt1 = (size_t)n_tiles + 1;
  const size_t ns = want_s ? (size_t)(n_src * S) : 0, nr = want_r ? (size_t)(n_rec * S) : 0;
  const size_t words = (want_s ? 2 * nt1 + 2 * ns : 0) + (want_r ? 2 * nt1 + 2 * nr : 0);
  const int n_rows = pt.tiles_y * (int)S;
  if (TB_CUDA(pool_malloc(reinterpret_cast<void **>(&ps.mem),
                          words * sizeof(int) + (size_t)n_rows, st)))
    return false;
  int *w = static_cast<int *>(ps.mem);
  if (want_s) {
    int *count = w, *start = w + nt1, *cell = w + 2 * nt1, *ent = w + 2 * nt1 + ns;
    if (!build_list(sources_i, (int)n_src, (int)S, L.g.N, L.g.nx, pt, n_tiles, count, start,
                    cell, ent, st, ps.src))
      return false;
    w += 2 * nt1 + 2 * ns;
  }
  if (want_r) {
    int *count = w, *start = w + nt1, *cell = w + 2 * nt1, *ent = w + 2 * nt1 + nr;
    if (!build_list(receivers_i, (int)n_rec, (int)S, L.g.N, L.g.nx, pt, n_tiles, count, start,
                    cell, ent, st, ps.rec))
      return false;
  }
  unsigned char *rowf = reinterpret_cast<unsigned char *>(static_cast<int *>(ps.mem) + words);
  k_points_rowflags<<<(n_rows + 255) / 256, 256, 0, st>>>(ps.src.start, ps.rec.start, pt.tiles_x,
                                                          n_rows, rowf);
  count_launches(1);
  ps.rowf = rowf;
  return !TB_CUDA(cudaGetLastError());
}


// ---------------------------------------------------------------------------
// Stencil order 2 runs the single-path kernels of tm2d_s2.cuh (Debye media use
// the generic E kernel); higher orders run the generic kernels.
template <typename T, int ST, typename S>
inline void launch_fwd_e(const Launch<T, ST> &L, cudaStream_t st, const T *ca, const T *cb,
                         const T *hx, const T *hz, T *ey, T *m_hx_z, T *m_hz_x, S *e_st,
                         S *c_st, const DebyeArgs<T> &db, const PointScratch &ps, const T *ft,
                         T *rt, const StepShift &sh = StepShift{}) {
  constexpr int NB = Launch<T, ST>::kNarrowBY;
  if (ST == 2 && db.n_poles == 0 && L.e_by == NB)
    k2_fwd_e<T, S, kRowsE, NB><<<L.grid_e_n, dim3(kTileX, NB, 1), 0, st>>>(
        L.g, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, e_st, c_st, ps.src, ps.rec, ft, rt, sh);
  else if (ST == 2 && db.n_poles == 0)
    k2_fwd_e<T, S, kRowsE><<<L.grid_e, L.block, 0, st>>>(L.g, ca, cb, hx, hz, ey, m_hx_z, m_hz_x,
                                                         e_st, c_st, ps.src, ps.rec, ft, rt, sh);
  else if (L.e_by == NB)
    k_fwd_e<T, ST, S, kRowsE, NB><<<L.grid_e_n, dim3(kTileX, NB, 1), 0, st>>>(
        L.g, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, e_st, c_st, db, ps.src, ps.rec, ft, rt, sh);
  else
    k_fwd_e<T, ST, S, kRowsE><<<L.grid_e, L.block, 0, st>>>(L.g, ca, cb, hx, hz, ey, m_hx_z,
                                                            m_hz_x, e_st, c_st, db, ps.src,
                                                            ps.rec, ft, rt, sh);
}

template <typename T, int ST>
inline void launch_fwd_h(const Launch<T, ST> &L, cudaStream_t st, const T *cq, const T *ey,
                         T *hx, T *hz, T *m_ey_x, T *m_ey_z) {
  if (ST == 2)
    k2_fwd_h<T, kRowsH><<<L.grid_h, L.block, 0, st>>>(L.g, cq, ey, hx, hz, m_ey_x, m_ey_z);
  else
    k_fwd_h<T, ST, kRowsH><<<L.grid_h, L.block, 0, st>>>(L.g, cq, ey, hx, hz, m_ey_x, m_ey_z);
}

template <typename T, int ST>
inline void launch_adj_e(const Launch<T, ST> &L, cudaStream_t st, const T *cb, const T *lam,
                         T *lhx, T *lhz, const T *mz, const T *mx, T *mz_n, T *mx_n) {
  constexpr int NB = Launch<T, ST>::kNarrowBY;
  if (ST == 2 && L.ae_by == NB)
    k2_adj_e<T, kRowsAE, NB><<<L.grid_ae_n, dim3(kTileX, NB, 1), 0, st>>>(L.g, cb, lam, lhx, lhz,
                                                                          mz, mx, mz_n, mx_n);
  else if (ST == 2)
    k2_adj_e<T, kRowsAE><<<L.grid_ae, L.block, 0, st>>>(L.g, cb, lam, lhx, lhz, mz, mx, mz_n,
                                                        mx_n);
  else if (L.ae_by == NB)
    k_adj_e<T, ST, kRowsAE, NB><<<L.grid_ae_n, dim3(kTileX, NB, 1), 0, st>>>(L.g, cb, lam, lhx,
                                                                             lhz, mz, mx, mz_n,
                                                                             mx_n);
  else
    k_adj_e<T, ST, kRowsAE><<<L.grid_ae, L.block, 0, st>>>(L.g, cb, lam, lhx, lhz, mz, mx, mz_n,
                                                           mx_n);
}

template <typename T, int ST, typename S>
inline void launch_adj_h(const Launch<T, ST> &L, cudaStream_t st, const T *ca, const T *cq,
                         const T *lhx, const T *lhz, T *ley, const T *mex, const T *mez,
                         T *mex_n, T *mez_n, const PointScratch &ps, const T *grt, T *gft,
                         const GradArgs<T, S> &ga, const StepShift &sh = StepShift{}) {
  if (ST == 2 && L.ah_by == 4)
    k2_adj_h<T, S, kRowsAH, 4><<<L.grid_ah, dim3(kTileX, 4, 1), 0, st>>>(
        L.g, ca, cq, lhx, lhz, ley, mex, mez, mex_n, mez_n, ps.rec, ps.src, ps.rowf, grt, gft, ga,
        sh);
  else if (ST == 2)
    k2_adj_h<T, S, kRowsAH, kBlockY><<<L.grid_ah, L.block, 0, st>>>(
        L.g, ca, cq, lhx, lhz, ley, mex, mez, mex_n, mez_n, ps.rec, ps.src, ps.rowf, grt, gft, ga,
        sh);
  else
    k_adj_h<T, ST, S, kRowsAH><<<L.grid_ah, L.block, 0, st>>>(L.g, ca, cq, lhx, lhz, ley, mex,
                                                              mez, mex_n, mez_n, ps.rec, ps.src,
                                                              grt, gft, ga, sh);
}

// ---------------------------------------------------------------------------
// Step blocks replayed from a CUDA graph.  A time step of the per-cell-kernel
// paths is two launches of 25-50 us each, and every launch costs the host a
// few microseconds; a host that falls behind leaves the GPU idle between
// steps.  So a long call runs its first block of steps as ordinary launches,
// captures the second block into a graph meanwhile (on a private stream:
// nothing runs during the capture) and replays that graph for every later
// block, one host call per block.  The step-indexed pointers of the captured
// launches (source and receiver rows, snapshot slots) move with a device word
// that the block's last launch advances (StepShift).  The block length is
// even and a multiple of the snapshot interval, so the steps that store or
// image a snapshot and the ping-pong state of the adjoint's CPML memories are
// the same in every block.  The steps after the last whole block run as
// ordinary launches.  With profiling on, a second graph of the block carries
// event-record nodes around the kernels of its first step and replays for
// the blocks that hold a profiled step (ProfileScope::arm gives it fresh
// events each time), so the sampled kernel times are those of graph-launched
// kernels; the ordinary launches of such a call are not sampled.
std::atomic<int> g_step_graphs{1};          // tide_b200_set_step_graphs
std::atomic<int64_t> g_graph_replays{0};    // tide_b200_graph_replays

__global__ void k_block_advance(int64_t *blk) { *blk += 1; }

// Steps per block when the step pattern repeats every `period` steps; 0: no
// graph (a block would exceed 256 steps).
inline int64_t graph_block_len(int64_t period) {
  const int64_t p = period % 2 ? 2 * period : period;  // lcm(2, period)
  if (p < 1 || p > 256) return 0;
  return ((64 + p - 1) / p) * p;
}

struct GraphHold {
  cudaStream_t st = nullptr, cs = nullptr;
  cudaGraph_t timed_graph = nullptr;  // kept: its event nodes are re-armed per replay
  cudaGraphExec_t exec = nullptr, timed = nullptr;
  int64_t *blk = nullptr;
  ~GraphHold() {
    if (exec) cudaGraphExecDestroy(exec);  // freed once its replays have run
    if (timed) cudaGraphExecDestroy(timed);
    if (timed_graph) cudaGraphDestroy(timed_graph);
    if (cs) cudaStreamDestroy(cs);
    if (blk) cudaFreeAsync(blk, st);
  }
};

// Captures steps [B, 2B) and the block advance into a graph on gh.cs; with
// `timed`, the first step's kernels are bracketed by the profile's
// event-record nodes.
template <typename Step>
bool capture_block(GraphHold &gh, int64_t B, Step &step, ProfileScope &prof, bool timed,
                   cudaGraph_t *graph) {
  *graph = nullptr;
  if (TB_CUDA(cudaStreamBeginCapture(gh.cs, cudaStreamCaptureModeThreadLocal))) return false;
  if (timed) prof.capture_begin(gh.cs);
  bool ok = true;
  for (int64_t i = B; i < 2 * B && ok; ++i) ok = step(i, gh.cs, gh.blk, B, timed && i == B);
  if (timed) prof.capture_end();
  if (ok) k_block_advance<<<1, 1, 0, gh.cs>>>(gh.blk);
  const cudaError_t ec = cudaStreamEndCapture(gh.cs, graph);
  if (!ok || TB_CUDA(ec)) {
    if (*graph) cudaGraphDestroy(*graph);
    *graph = nullptr;
    return false;
  }
  return true;
}

// Runs steps 0..n-1 of a call.  step(i, stream, blk, B, smp) launches step i
// on `stream`, with profiling events when smp; blk != nullptr marks a
// captured launch (StepShift over blocks of B steps).  A block is profiled
// when prof samples one of its steps.
template <typename Step>
bool run_step_blocks(int64_t n, int64_t period, cudaStream_t st, ProfileScope &prof,
                     int64_t (*t_of)(int64_t, int64_t), int64_t t_base, Step &&step) {
  auto sampled = [&](int64_t i) { return prof.sample(t_of(t_base, i)); };
  const int64_t B = g_step_graphs.load() ? graph_block_len(period) : 0;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (B > 0 && n >= 3 * B && TB_CUDA(cudaStreamIsCapturing(st, &cap))) return false;
  if (B == 0 || n < 3 * B || cap != cudaStreamCaptureStatusNone) {
    for (int64_t i = 0; i < n; ++i)
      if (!step(i, st, nullptr, B, sampled(i))) return false;
    return true;
  }
  // Block 0 runs while block 1 is captured.  Profiled steps outside the
  // replayed blocks (block 0, the tail) are not timed: only graph-launched
  // kernels are sampled on this path.
  for (int64_t i = 0; i < B; ++i)
    if (!step(i, st, nullptr, B, false)) return false;
  GraphHold gh;
  gh.st = st;
  if (TB_CUDA(pool_malloc((void **)&gh.blk, sizeof(int64_t), st))) return false;
  if (TB_CUDA(cudaMemsetAsync(gh.blk, 0, sizeof(int64_t), st))) return false;
  if (TB_CUDA(cudaStreamCreateWithFlags(&gh.cs, cudaStreamNonBlocking))) return false;
  cudaGraph_t graph = nullptr;
  if (!capture_block(gh, B, step, prof, false, &graph)) return false;
  const cudaError_t ei = cudaGraphInstantiate(&gh.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (TB_CUDA(ei)) return false;
  if (prof.on()) {
    if (!capture_block(gh, B, step, prof, true, &gh.timed_graph)) return false;
    if (prof.bind(gh.timed_graph) &&
        TB_CUDA(cudaGraphInstantiate(&gh.timed, gh.timed_graph, 0)))
      return false;
  }
  const int64_t nb = n / B;
  for (int64_t b = 1; b < nb; ++b) {
    bool smp = false;
    for (int64_t i = b * B; i < (b + 1) * B && !smp; ++i) smp = sampled(i);
    const cudaGraphExec_t ge = smp && gh.timed && prof.arm(gh.timed) ? gh.timed : gh.exec;
    if (TB_CUDA(cudaGraphLaunch(ge, st))) return false;
    g_graph_replays.fetch_add(1, std::memory_order_relaxed);
  }
  count_launches(nb - 1);  // block advances
  for (int64_t i = nb * B; i < n; ++i)
    if (!step(i, st, nullptr, B, false)) return false;
  return !TB_CUDA(cudaGetLastError());
}
inline int64_t t_up(int64_t t0, int64_t i) { return t0 + i; }
inline int64_t t_down(int64_t t0, int64_t i) { return t0 - 1 - i; }

// ---------------------------------------------------------------------------
// Fused stencil-2 FP32 forward (tm2d_fused.cuh) on a pitched internal copy of
// the state: two copies of Ey, Hx, Hz, m_ey_x, m_ey_z (ping-pong), one of
// m_hx_z, m_hz_x (updated in place) and of the coefficients, every array with
// a guard row before and after it.  The copy is made at the start of a call
// and the final state copied back at its end.
struct PitchedFwd {
  void *mem = nullptr;
  cudaStream_t st = nullptr;
  F4Geom q{};
  int nx = 0;
  float *cur[5] = {}, *nxt[5] = {}, *mhx = nullptr, *mhz = nullptr;
  float *ca = nullptr, *cb = nullptr, *cq = nullptr;
  float *user[7] = {};  // caller's ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x
  int64_t rows = 0;     // rows of the state arrays (n_shots * ny)
  ~PitchedFwd() {
    if (mem) cudaFreeAsync(mem, st);
  }
  // Pitched array base points at row 0, pitched column 0 (column x at + padl).
  bool copy_in(float *dst, const float *src, int64_t nrows) {
    return !TB_CUDA(cudaMemcpy2DAsync(dst + q.padl, (size_t)q.pitch * 4, src, (size_t)nx * 4,
                                      (size_t)nx * 4, (size_t)nrows, cudaMemcpyDeviceToDevice,
                                      st));
  }
  // Device bytes of the pitched copy of geometry g (state, memories,
  // coefficients, guard rows).
  static size_t bytes_for(const TMGeom<float> &g) {
    const F4Geom q = f4_geom(g);
    const int64_t rows = (int64_t)g.n_shots * g.ny;
    size_t total = 12 * (size_t)(rows + 2) * q.pitch;
    const int64_t rc[3] = {(g.ca_b ? g.n_shots : 1) * (int64_t)g.ny,
                           (g.cb_b ? g.n_shots : 1) * (int64_t)g.ny,
                           (g.cq_b ? g.n_shots : 1) * (int64_t)g.ny};
    for (int i = 0; i < 3; ++i) total += (size_t)(rc[i] + 2) * q.pitch;
    return total * sizeof(float);
  }
  bool init(const TMGeom<float> &g, float *const fields[7], const float *ca_u,
            const float *cb_u, const float *cq_u, cudaStream_t s) {
    st = s;
    nx = g.nx;
    q = f4_geom(g);
    if (q.pshot > ((int64_t)1 << 31) - 1 - 2 * q.pitch) {
      set_error(kBadArgument, "TM2D: ny * pitch too large for the fused forward");
      return false;
    }
    rows = (int64_t)g.n_shots * g.ny;
    const int64_t rc[3] = {(g.ca_b ? g.n_shots : 1) * (int64_t)g.ny,
                           (g.cb_b ? g.n_shots : 1) * (int64_t)g.ny,
                           (g.cq_b ? g.n_shots : 1) * (int64_t)g.ny};
    const size_t state = (size_t)(rows + 2) * q.pitch;
    const size_t total = bytes_for(g) / sizeof(float);
    if (TB_CUDA(pool_malloc(&mem, total * sizeof(float), st))) return false;
    if (TB_CUDA(cudaMemsetAsync(mem, 0, total * sizeof(float), st))) return false;
    float *p = static_cast<float *>(mem);
    auto take = [&](size_t n) {
      float *r = p + q.pitch;  // past the leading guard row
      p += n;
      return r;
    };
    for (int i = 0; i < 5; ++i) cur[i] = take(state);
    for (int i = 0; i < 5; ++i) nxt[i] = take(state);
    mhx = take(state);
    mhz = take(state);
    ca = take((size_t)(rc[0] + 2) * q.pitch);
    cb = take((size_t)(rc[1] + 2) * q.pitch);
    cq = take((size_t)(rc[2] + 2) * q.pitch);
    for (int i = 0; i < 7; ++i) user[i] = fields[i];
    for (int i = 0; i < 5; ++i)
      if (!copy_in(cur[i], user[i], rows) || !copy_in(nxt[i], user[i], rows)) return false;
    return copy_in(mhx, user[5], rows) && copy_in(mhz, user[6], rows) &&
           copy_in(ca, ca_u, rc[0]) && copy_in(cb, cb_u, rc[1]) && copy_in(cq, cq_u, rc[2]);
  }
  // State of the next step (old = current copy, new = the other); swaps.
  FwdState<float> step() {
    const FwdState<float> fs{cur[0], cur[1], cur[2], cur[3], cur[4], mhx, mhz,
                             nxt[0], nxt[1], nxt[2], nxt[3], nxt[4], mhx, mhz};
    for (int i = 0; i < 5; ++i) std::swap(cur[i], nxt[i]);
    return fs;
  }
  bool finish() {
    const float *fin[7] = {cur[0], cur[1], cur[2], cur[3], cur[4], mhx, mhz};
    for (int i = 0; i < 7; ++i)
      if (TB_CUDA(cudaMemcpy2DAsync(user[i], (size_t)nx * 4, fin[i] + q.padl,
                                    (size_t)q.pitch * 4, (size_t)nx * 4, (size_t)rows,
                                    cudaMemcpyDeviceToDevice, st)))
        return false;
    return true;
  }
  // One time step (one launch).
  template <typename S_>
  void launch(const TMGeom<float> &g, S_ *e_st, S_ *c_st, const PointScratch &ps,
              const float *ft, float *rt) {
    const F4Blocks nb = f4_blocks(q);
    const dim3 grid((unsigned)(nb.n_side + nb.n_band + nb.n_int), 1, (unsigned)g.n_shots);
    f4_fwd_step<S_><<<grid, dim3(32, kF4Warps, 1), 0, st>>>(g, q, nb, ca, cb, cq, step(), e_st,
                                                            c_st, ps.src, ps.rec, ps.rowf, ft,
                                                            rt);
  }
};

template <typename T> constexpr bool is_float() { return std::is_same<T, float>::value; }

// ---------------------------------------------------------------------------
// One-sweep TMA path (tm2d_tma.cuh): FP32, stencil 2, model coefficients
// shared by the shots, no Debye poles.  A call copies its fields into two
// pitched copies (ping-pong) and its coefficients into a pitched copy,
// encodes the tensor maps of both copies once, runs one launch per time
// step on P = min(SMs, tiles) persistent CTAs and copies the final state
// back.  Mode (tide_b200_set_tma_mode): 0 off (default: on the 553 x 1065,
// 8-shot gradient workload these kernels issue about 270 instructions per
// cell and run slower than the per-call pair kernels), 1 when the grid has
// at least kQMinTiles tiles, 2 whenever eligible.
std::atomic<int> g_tma_mode{0};
std::atomic<int> g_tma_max_ctas{0};  // 0: one CTA per SM (tide_b200_set_tma_ctas)
constexpr int kQTY = 32;        // tile height of the TMA kernels
constexpr int kQMinTiles = 64;  // auto mode: below this the per-call kernels win

template <bool ADJ> struct QRun {
  using B = QBox;
  cudaStream_t st = nullptr;
  void *mem = nullptr;
  int64_t pitch = 0, pshot = 0;
  int nx = 0, ny = 0, S = 0, tiles_x = 0, tiles_y = 0, P = 0;
  float *f[2][3] = {};  // pitched copies [set][Ey, Hx, Hz]
  float *coef[3] = {};  // adjoint: ca, cb, cq; forward: cq, ca, cb
  float *user[3] = {};  // caller's field arrays
  QMaps maps[2];
  int cur = 0;
  // forward: H-phase memories ping-pong (caller's array and a copy)
  float *mex[2] = {}, *mez[2] = {};
  float *user_mex = nullptr, *user_mez = nullptr;
  // adjoint: hand-off sums and flags
  float *hand = nullptr;
  int *flags = nullptr;
  int *order = nullptr;  // grid tile at each position of the tile sequence
  int epoch = 0;
  ~QRun() {
    if (mem) cudaFreeAsync(mem, st);
  }

  static bool eligible(const TMGeom<float> &g, int64_t nt) {
    const int mode = g_tma_mode.load();
    if (mode == 0 || nt <= 0 || g.ca_b || g.cb_b || g.cq_b) return false;
    if (g.nx < 2 || g.ny < 2) return false;
    const int64_t tiles = (int64_t)((g.nx + kQX - 1) / kQX) * ((g.ny + kQTY - 1) / kQTY);
    if ((int64_t)g.n_shots * tiles > ((int64_t)1 << 30)) return false;
    return mode == 2 || tiles >= kQMinTiles;
  }

  bool copy2d(float *dst, int64_t dpitch, const float *src, int64_t spitch, int64_t rows) {
    return !TB_CUDA(cudaMemcpy2DAsync(dst, (size_t)dpitch * 4, src, (size_t)spitch * 4,
                                      (size_t)nx * 4, (size_t)rows, cudaMemcpyDeviceToDevice, st));
  }

  // fields: caller's Ey, Hx, Hz (or lambda_*); c3: adjoint ca, cb, cq /
  // forward cq, ca, cb; mex / mez: forward H-phase memories (null for the
  // adjoint).
  bool init(const TMGeom<float> &g, float *const fields[3], const float *const c3[3],
            float *m_ey_x, float *m_ey_z, cudaStream_t s) {
    st = s;
    nx = g.nx; ny = g.ny; S = g.n_shots;
    pitch = ((int64_t)nx + 31) / 32 * 32;
    pshot = (int64_t)ny * pitch;
    tiles_x = (nx + kQX - 1) / kQX;
    tiles_y = (ny + kQTY - 1) / kQTY;
    int dev = 0, n_sm = 0;
    if (TB_CUDA(cudaGetDevice(&dev)) ||
        TB_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)))
      return false;
    const int cap = g_tma_max_ctas.load();
    P = std::max(1, std::min(cap > 0 ? std::min(cap, n_sm) : n_sm, tiles_x * tiles_y));
    const size_t state = (size_t)S * (size_t)pshot;
    const size_t N = (size_t)ny * nx;
    const int tiles = tiles_x * tiles_y;
    size_t total = 6 * state + 3 * (size_t)pshot + (size_t)tiles;
    if (ADJ) total += (size_t)P * 2 * kQTY * kQX + (size_t)P;
    else total += 2 * (size_t)S * N;
    if (TB_CUDA(pool_malloc(&mem, total * sizeof(float), st))) return false;
    float *p = static_cast<float *>(mem);
    for (int k = 0; k < 2; ++k)
      for (int i = 0; i < 3; ++i) {
        f[k][i] = p;
        p += state;
      }
    for (int i = 0; i < 3; ++i) {
      coef[i] = p;
      p += pshot;
    }
    order = reinterpret_cast<int *>(p);
    p += tiles;
    if (!upload_order(g)) return false;
    for (int i = 0; i < 3; ++i) {
      user[i] = fields[i];
      if (!copy2d(f[0][i], pitch, fields[i], nx, (int64_t)S * ny)) return false;
      if (!copy2d(coef[i], pitch, c3[i], nx, ny)) return false;
    }
    if (ADJ) {
      hand = p;
      p += (size_t)P * 2 * kQTY * kQX;
      flags = reinterpret_cast<int *>(p);
      if (TB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * (size_t)P, st))) return false;
    } else {
      user_mex = m_ey_x; user_mez = m_ey_z;
      mex[0] = m_ey_x; mez[0] = m_ey_z;
      mex[1] = p; p += (size_t)S * N;
      mez[1] = p; p += (size_t)S * N;
      // the copies start equal, so cells outside the strips (never written)
      // agree in both
      if (TB_CUDA(cudaMemcpyAsync(mex[1], m_ey_x, S * N * 4, cudaMemcpyDeviceToDevice, st)) ||
          TB_CUDA(cudaMemcpyAsync(mez[1], m_ey_z, S * N * 4, cudaMemcpyDeviceToDevice, st)))
        return false;
    }
    for (int k = 0; k < 2; ++k) {
      QMaps &m = maps[k];
      if (!encode_map_3d(&m.e, f[k][0], nx, ny, S, pitch, B::EW, B::EH) ||
          !encode_map_3d(&m.x, f[k][1], nx, ny, S, pitch, B::XW, B::XH) ||
          !encode_map_3d(&m.z, f[k][2], nx, ny, S, pitch, B::ZW, B::ZH))
        return false;
      if (ADJ) {
        if (!encode_map_3d(&m.c0, coef[0], nx, ny, 1, pitch, B::OW, B::OH) ||
            !encode_map_3d(&m.c1, coef[1], nx, ny, 1, pitch, B::EW, B::EH) ||
            !encode_map_3d(&m.c2, coef[2], nx, ny, 1, pitch, B::QW, B::QH))
          return false;
      } else {
        if (!encode_map_3d(&m.c0, coef[0], nx, ny, 1, pitch, B::QW, B::QH) ||
            !encode_map_3d(&m.c1, coef[1], nx, ny, 1, pitch, B::OW, B::OH) ||
            !encode_map_3d(&m.c2, coef[2], nx, ny, 1, pitch, B::OW, B::OH))
          return false;
      }
    }
    return true;
  }

  // Tile sequence: tiles that take the CPML / edge path are spread evenly
  // between the interior ones (tile k of a class of n goes to key (k+0.5)/n),
  // so every CTA's contiguous range of units holds the same mix.
  bool upload_order(const TMGeom<float> &g) {
    const int tiles = tiles_x * tiles_y;
    std::vector<std::pair<double, int>> key;
    key.reserve(tiles);
    int n_cls[2] = {0, 0};
    std::vector<int> cls(tiles);
    for (int t = 0; t < tiles; ++t) {
      const int y0 = (t / tiles_x) * kQTY, x0 = (t % tiles_x) * kQX;
      const bool in = y0 - 1 >= std::max(1, g.pml_y0) && y0 + kQTY < std::min(g.ny, g.pml_y1) &&
                      x0 - 1 >= std::max(1, g.pml_x0) && x0 + kQX < std::min(g.nx, g.pml_x1);
      cls[t] = in ? 0 : 1;
      ++n_cls[cls[t]];
    }
    int seen[2] = {0, 0};
    for (int t = 0; t < tiles; ++t) {
      const int c = cls[t];
      key.emplace_back((seen[c]++ + 0.5) / n_cls[c] + 1e-9 * c, t);
    }
    std::stable_sort(key.begin(), key.end());
    std::vector<int> h(tiles);
    for (int t = 0; t < tiles; ++t) h[t] = key[t].second;
    return !TB_CUDA(cudaMemcpyAsync(order, h.data(), sizeof(int) * tiles,
                                    cudaMemcpyHostToDevice, st)) &&
           !TB_CUDA(cudaStreamSynchronize(st));
  }

  QCommon common(const TMGeom<float> &g, const PointScratch &ps, const float *va,
                 float *vb) const {
    QCommon c{};
    c.g = g;
    c.tiles_x = tiles_x; c.tiles_y = tiles_y; c.P = P;
    c.order = order;
    c.pitch = pitch; c.pshot = pshot;
    c.ey_n = f[cur ^ 1][0]; c.hx_n = f[cur ^ 1][1]; c.hz_n = f[cur ^ 1][2];
    c.pa = ADJ ? ps.rec : ps.src;
    c.pb = ADJ ? ps.src : ps.rec;
    c.va = va; c.vb = vb;
    return c;
  }

  // Opt the kernel into its dynamic shared memory once per device.
  template <typename SN> bool prepare() const {
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    if (TB_CUDA(cudaGetDevice(&dev))) return false;
    const uint64_t bit = uint64_t(1) << (dev & 63);
    if (done.load() & bit) return true;
    const cudaError_t e =
        ADJ ? cudaFuncSetAttribute(kq_adj_step<SN>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   B::smem_bytes(true))
            : cudaFuncSetAttribute(kq_fwd_step<SN>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   B::smem_bytes(false));
    if (TB_CUDA(e)) return false;
    done.fetch_or(bit);
    return true;
  }

  // One forward step: E-phase memories m_hx_z / m_hz_x in place.
  template <typename SN>
  bool fwd_step(const TMGeom<float> &g, const PointScratch &ps, const float *ft, float *rt,
                float *mhx, float *mhz, SN *e_st, SN *c_st) {
    if (!prepare<SN>()) return false;
    QFwdArgs a{};
    a.c = common(g, ps, ft, rt);
    a.mex_c = mex[cur]; a.mez_c = mez[cur];
    a.mex_n = mex[cur ^ 1]; a.mez_n = mez[cur ^ 1];
    a.mhx = mhx; a.mhz = mhz;
    a.ey_st = e_st; a.cu_st = c_st;
    kq_fwd_step<SN><<<P, kQThreads, B::smem_bytes(false), st>>>(maps[cur], a);
    cur ^= 1;
    return true;
  }

  // One adjoint step; mem_c / mem_n: the l-memories (hz_x, hx_z, ey_x, ey_z)
  // read / written.
  template <typename SN>
  bool adj_step(const TMGeom<float> &g, const PointScratch &ps, const float *grt, float *gft,
                const float *const mem_c[4], float *const mem_n[4], const SN *e_st,
                const SN *c_st, int bg_shots, float *grad_ca, float *grad_cb, float kscale) {
    if (!prepare<SN>()) return false;
    QAdjArgs a{};
    a.c = common(g, ps, grt, gft);
    a.mhz_c = mem_c[0]; a.mhx_c = mem_c[1]; a.mex_c = mem_c[2]; a.mez_c = mem_c[3];
    a.mhz_n = mem_n[0]; a.mhx_n = mem_n[1]; a.mex_n = mem_n[2]; a.mez_n = mem_n[3];
    a.ey_st = e_st; a.cu_st = c_st;
    a.bg_shots = bg_shots;
    a.grad_ca = grad_ca; a.grad_cb = grad_cb;
    a.kscale = kscale;
    a.hand = hand; a.flags = flags;
    a.epoch = ++epoch;
    kq_adj_step<SN><<<P, kQThreads, B::smem_bytes(true), st>>>(maps[cur], a);
    cur ^= 1;
    return true;
  }

  // Copy the final state back into the caller's arrays.
  bool finish() {
    for (int i = 0; i < 3; ++i)
      if (!copy2d(user[i], nx, f[cur][i], pitch, (int64_t)S * ny)) return false;
    if (!ADJ && mex[cur] != user_mex) {
      const size_t nb = (size_t)S * ny * nx * 4;
      if (TB_CUDA(cudaMemcpyAsync(user_mex, mex[cur], nb, cudaMemcpyDeviceToDevice, st)) ||
          TB_CUDA(cudaMemcpyAsync(user_mez, mez[cur], nb, cudaMemcpyDeviceToDevice, st)))
        return false;
    }
    return true;
  }
  PointTiles point_tiles() const { return PointTiles{tiles_x, tiles_y, kQX, kQTY, 0}; }
};


// The two-kernel forward re-reads H and Ey between its half steps; while the
// three fields of a call fit in about half of the 126 MB L2 those re-reads
// are L2 hits and the two-kernel path is the faster one (measured on the
// 553 x 1065 grid: 8 shots two-kernel 51.8 us/step vs fused 55.8; 24 shots
// fused 134 vs two-kernel 171).  Above that the fused step's single HBM
// sweep wins.
std::atomic<int64_t> g_fused_min_bytes{(int64_t)64 << 20};  // tide_b200_set_fused_threshold
inline bool fused_pays(int64_t n_shots, int64_t cells) {
  const int64_t t = g_fused_min_bytes.load();
  return t >= 0 && 3 * n_shots * cells * (int64_t)sizeof(float) > t;
}

template <typename T, int ST>
void tm_forward(TIDE_TM_FORWARD_ARGS(T)) {
  (void)dt; (void)step_ratio; (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0, "TM2D forward: nt must be >= 0");
  TB_REQUIRE(ca && cb && cq && ey && hx && hz && m_ey_x && m_ey_z && m_hx_z && m_hz_x,
             "TM2D forward: a field or coefficient pointer is null");
  TB_REQUIRE(n_sources_per_shot == 0 || f, "TM2D forward: sources without amplitudes");
  TB_REQUIRE(n_receivers_per_shot == 0 || r, "TM2D forward: receivers without output");
  DebyeArgs<T> db{nullptr, nullptr, nullptr, nullptr, 0};
  if (has_dispersion) {
    TB_REQUIRE(n_poles >= 1 && debye_a && debye_b && debye_cp && polarization,
               "TM2D forward: dispersion enabled without Debye coefficients");
    db = DebyeArgs<T>{debye_a, debye_b, debye_cp, polarization, (int)n_poles};
  }
  (void)ey_prev;  // the old Ey lives in a register; the buffer is not needed
  Launch<T, ST> L;
  if (!make_launch(L, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, rdy, rdx, n_shots,
                   ny, nx, pml_y0, pml_x0, pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  cudaStream_t st = as_stream(compute_stream);
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  if constexpr (is_float<T>() && ST == 2) {
    if (db.n_poles == 0 && L.has_domain && QRun<false>::eligible(L.g, nt)) {
      // One-sweep TMA path.
      QRun<false> qr;
      float *const fl[3] = {ey, hx, hz};
      const float *const c3[3] = {cq, ca, cb};
      if (!qr.init(L.g, fl, c3, m_ey_x, m_ey_z, st)) return;
      PointScratch ps;
      if (!build_points(ps, L, qr.point_tiles(), sources_i, n_sources_per_shot, receivers_i,
                        n_receivers_per_shot, st))
        return;
      ProfileScope prof(st);
      for (int64_t t = start_t; t < start_t + nt; ++t) {
        const bool smp = prof.sample(t);
        if (smp) prof.begin(kKFwdStep);
        if (!qr.template fwd_step<float>(L.g, ps, f ? f + t * fs : nullptr,
                                         r ? r + t * rs : nullptr, m_hx_z, m_hz_x, nullptr,
                                         nullptr))
          return;
        if (smp) prof.end(kKFwdStep);
      }
      count_launches(nt);
      if (TB_CUDA(cudaGetLastError())) return;
      qr.finish();
      return;
    }
    if (db.n_poles == 0 && L.has_domain && nt > 0 && fused_pays(n_shots, L.g.N)) {
      // Fused one-launch-per-step path.
      PitchedFwd pf;
      float *const fields[7] = {ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x};
      if (!pf.init(L.g, fields, ca, cb, cq, st)) return;
      PointScratch ps;
      if (!build_points(ps, L, pf.q.pt, sources_i, n_sources_per_shot, receivers_i,
                        n_receivers_per_shot, st))
        return;
      ProfileScope prof(st);
      for (int64_t t = start_t; t < start_t + nt; ++t) {
        const bool smp = prof.sample(t);
        if (smp) prof.begin(kKFwdStep);
        pf.launch<float>(L.g, nullptr, nullptr, ps, f ? f + t * fs : nullptr,
                         r ? r + t * rs : nullptr);
        if (smp) prof.end(kKFwdStep);
      }
      count_launches(nt);
      if (TB_CUDA(cudaGetLastError())) return;
      pf.finish();
      return;
    }
  }
  if (db.n_poles == 0) L.narrow_e();
  PointScratch ps;
  if (!build_points(ps, L, L.e_tiles(), sources_i, n_sources_per_shot, receivers_i,
                    n_receivers_per_shot, st))
    return;
  ProfileScope prof(st);
  auto step = [&](int64_t i, cudaStream_t s, const int64_t *blk, int64_t B, bool smp) -> bool {
    const int64_t t = start_t + i;
    if (L.has_domain) {
      if (smp) prof.begin(kKFwdH);
      launch_fwd_h<T, ST>(L, s, cq, ey, hx, hz, m_ey_x, m_ey_z);
      if (smp) prof.end(kKFwdH);
    }
    if (smp) prof.begin(kKFwdE);
    launch_fwd_e<T, ST, T>(L, s, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, nullptr, nullptr, db, ps,
                           f ? f + t * fs : nullptr, r ? r + t * rs : nullptr,
                           StepShift{blk, B * fs, B * rs, 0});
    if (smp) prof.end(kKFwdE);
    return true;
  };
  if (!run_step_blocks(nt, 1, st, prof, t_up, start_t, step)) return;
  count_launches(nt * (L.has_domain ? 2 : 1));
  TB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
template <typename T, int ST>
void tm_forward_with_storage(TIDE_TM_FORWARD_WITH_STORAGE_ARGS(T)) {
  (void)dt; (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1, "TM2D forward_with_storage: bad nt/step_ratio");
  TB_REQUIRE(ca && cb && cq && ey && hx && hz && m_ey_x && m_ey_z && m_hx_z && m_hz_x,
             "TM2D forward_with_storage: a field or coefficient pointer is null");
  TB_REQUIRE(n_sources_per_shot == 0 || f, "TM2D forward_with_storage: sources without amplitudes");
  TB_REQUIRE(n_receivers_per_shot == 0 || r, "TM2D forward_with_storage: receivers without output");
  cudaStream_t st = as_stream(compute_stream);
  StoreRun<2> sr;
  {
    const bool need[2] = {ca_requires_grad, cb_requires_grad};
    void *const dev[2] = {ey_store_1, curl_store_1}, *const host[2] = {ey_store_3, curl_store_3};
    char const *const *const files[2] = {ey_filenames, curl_filenames};
    if (!sr.init("TM2D", need, storage_mode, storage_format, sizeof(T), shot_bytes_uncomp,
                 ny * nx, n_shots, step_ratio, dev, host, files, st, as_stream(storage_stream)))
      return;
  }
  Launch<T, ST> L;
  if (!make_launch(L, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, rdy, rdx, n_shots,
                   ny, nx, pml_y0, pml_x0, pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  // one launch per step: the TMA path, else the pitched fused path (see fused_pays)
  bool qpath = false;
  if constexpr (is_float<T>() && ST == 2) qpath = L.has_domain && QRun<false>::eligible(L.g, nt);
  const bool fused = !qpath && is_float<T>() && ST == 2 && L.has_domain && nt > 0 &&
                     fused_pays(n_shots, L.g.N);
  PitchedFwd pf;
  QRun<false> qr;
  if constexpr (is_float<T>()) {
    float *const fields[7] = {ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x};
    if (fused && !pf.init(L.g, fields, ca, cb, cq, st)) return;
    float *const fl[3] = {ey, hx, hz};
    const float *const c3[3] = {cq, ca, cb};
    if (qpath && !qr.init(L.g, fl, c3, m_ey_x, m_ey_z, st)) return;
  }
  if (!qpath && !fused) L.narrow_e();
  PointScratch ps;
  if (!(qpath   ? build_points(ps, L, qr.point_tiles(), sources_i, n_sources_per_shot,
                               receivers_i, n_receivers_per_shot, st)
        : fused ? build_points(ps, L, pf.q.pt, sources_i, n_sources_per_shot, receivers_i,
                               n_receivers_per_shot, st)
                : build_points(ps, L, L.e_tiles(), sources_i, n_sources_per_shot, receivers_i,
                               n_receivers_per_shot, st)))
    return;
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  const DebyeArgs<T> db{nullptr, nullptr, nullptr, nullptr, 0};
  const bool bf16 = sr.bf16;
  ProfileScope prof(st);
  if (!qpath && !fused) {
    // Per-cell kernels; with the history on the device the step blocks are
    // replayed from a graph (run_step_blocks).
    const int64_t snap = sr.want ? (int64_t)(sr.step_bytes / (bf16 ? 2 : sizeof(T))) : 0;
    auto step = [&](int64_t i, cudaStream_t s, const int64_t *blk, int64_t B, bool smp) -> bool {
      const int64_t t = start_t + i;
      const bool store_step = sr.stores(t);
      char *dst[2];
      if (!sr.begin(t, dst)) return false;
      char *const e1 = dst[0], *const c1 = dst[1];
      const T *ft = f ? f + t * fs : nullptr;
      T *rt = r ? r + t * rs : nullptr;
      const StepShift sh{blk, B * fs, B * rs, B / step_ratio * snap};
      if (L.has_domain) {
        if (smp) prof.begin(kKFwdH);
        launch_fwd_h<T, ST>(L, s, cq, ey, hx, hz, m_ey_x, m_ey_z);
        if (smp) prof.end(kKFwdH);
      }
      if (smp) prof.begin(kKFwdE);
      if (store_step && bf16)
        launch_fwd_e<T, ST, __nv_bfloat16>(L, s, ca, cb, hx, hz, ey, m_hx_z, m_hz_x,
                                           (__nv_bfloat16 *)e1, (__nv_bfloat16 *)c1, db, ps, ft,
                                           rt, sh);
      else
        launch_fwd_e<T, ST, T>(L, s, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, (T *)e1, (T *)c1, db,
                               ps, ft, rt, sh);
      if (smp) prof.end(kKFwdE);
      return sr.end(t, dst);
    };
    if (sr.host_side) {
      for (int64_t i = 0; i < nt; ++i)
        if (!step(i, st, nullptr, 0, prof.sample(start_t + i))) return;
    } else if (!run_step_blocks(nt, sr.want ? step_ratio : 1, st, prof, t_up, start_t, step)) {
      return;
    }
    count_launches(nt * (L.has_domain ? 2 : 1));
    if (TB_CUDA(cudaGetLastError())) return;
    sr.finish();
    return;
  }
  for (int64_t t = start_t; t < start_t + nt; ++t) {
    const bool smp = prof.sample(t);
    const bool store_step = sr.stores(t);
    char *dst[2];
    if (!sr.begin(t, dst)) return;
    char *const e1 = dst[0], *const c1 = dst[1];
    const T *ft = f ? f + t * fs : nullptr;
    T *rt = r ? r + t * rs : nullptr;
    if (qpath) {
      if (smp) prof.begin(kKFwdStep);
      if constexpr (is_float<T>()) {
        const bool ok =
            (store_step && bf16)
                ? qr.template fwd_step<__nv_bfloat16>(L.g, ps, ft, rt, m_hx_z, m_hz_x,
                                                      (__nv_bfloat16 *)e1, (__nv_bfloat16 *)c1)
                : qr.template fwd_step<float>(L.g, ps, ft, rt, m_hx_z, m_hz_x, (float *)e1,
                                              (float *)c1);
        if (!ok) return;
      }
      if (smp) prof.end(kKFwdStep);
    } else {
      if (smp) prof.begin(kKFwdStep);
      if constexpr (is_float<T>()) {
        if (store_step && bf16)
          pf.launch<__nv_bfloat16>(L.g, (__nv_bfloat16 *)e1, (__nv_bfloat16 *)c1, ps, ft, rt);
        else
          pf.launch<float>(L.g, (float *)e1, (float *)c1, ps, ft, rt);
      }
      if (smp) prof.end(kKFwdStep);
    }
    if (!sr.end(t, dst)) return;
  }
  count_launches(nt);
  if (TB_CUDA(cudaGetLastError())) return;
  if constexpr (is_float<T>()) {
    if (fused && !pf.finish()) return;
    if (qpath && !qr.finish()) return;
  }
  sr.finish();
}

// ---------------------------------------------------------------------------
template <typename T>
bool zero_band(T *m, const TMGeom<T> &g, int axis, int lo, int hi, cudaStream_t st) {
  if (hi <= lo) return true;
  k_zero_band<T><<<1184, 256, 0, st>>>(m, g.n_shots, g.ny, g.nx, axis, lo, hi);
  count_launches(1);
  return !TB_CUDA(cudaGetLastError());
}

// Exact adjoint (backward) and its background-reuse form: with
// background_n_shots < n_shots the snapshot history holds background_n_shots
// shots and adjoint shot s images against snapshot shot s %
// background_n_shots (maxwell_tm_cuda_inst.cu:2405-2460, 651-660).
template <typename T, int ST>
void tm_backward(TIDE_TM_BACKWARD_ARGS(T), int64_t background_n_shots) {
  (void)dt; (void)n_threads; (void)ey_filenames; (void)curl_filenames;
  (void)grad_ca_shot; (void)grad_cb_shot;  // gradients are reduced in-kernel (see k_adj_h)
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1 && start_t - nt >= 0,
             "TM2D backward: bad nt/step_ratio/start_t");
  TB_REQUIRE(ca && cb && cq && lambda_ey && lambda_hx && lambda_hz && m_lambda_ey_x &&
                 m_lambda_ey_z && m_lambda_hx_z && m_lambda_hz_x && adjoint_memory_scratch,
             "TM2D backward: a field or coefficient pointer is null");
  TB_REQUIRE(n_receivers_per_shot == 0 || grad_r, "TM2D backward: receivers without grad_r");
  TB_REQUIRE(background_n_shots >= 1 && n_shots % background_n_shots == 0,
             "TM2D backward: n_shots (%lld) must be a multiple of background_n_shots (%lld)",
             (long long)n_shots, (long long)background_n_shots);
  const int bg_shots = (int)background_n_shots;
  const bool bf16 = storage_format == 1;
  TB_REQUIRE(!bf16 || sizeof(T) == 4, "TM2D: bf16 snapshot storage requires float32 fields");
  const bool grads = (ca_requires_grad || cb_requires_grad) && storage_mode != 3;
  const size_t esz = bf16 ? 2 : sizeof(T);
  if (grads) {
    TB_REQUIRE(shot_bytes_uncomp == ny * nx * (int64_t)esz,
               "TM2D backward: shot_bytes_uncomp does not match ny*nx*elem");
    TB_REQUIRE((!ca_requires_grad || (ey_store_1 && grad_ca)) &&
                   (!cb_requires_grad || (curl_store_1 && grad_cb)),
               "TM2D backward: gradient or snapshot buffers missing");
    TB_REQUIRE((storage_mode != 1 && storage_mode != 2) ||
                   ((!ca_requires_grad || ey_store_3) && (!cb_requires_grad || curl_store_3)),
               "TM2D backward: cpu / disk storage modes need host snapshot buffers");
    TB_REQUIRE(storage_mode != 2 ||
                   ((!ca_requires_grad || (ey_filenames && ey_filenames[0])) &&
                    (!cb_requires_grad || (curl_filenames && curl_filenames[0]))),
               "TM2D backward: disk storage mode needs snapshot file names");
  }
  Launch<T, ST> L;
  if (!make_launch(L, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, rdy, rdx, n_shots,
                   ny, nx, pml_y0, pml_x0, pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  if constexpr (ST == 2) pick_adj_h_rows<T, T>(L);
  L.narrow_e();
  cudaStream_t st = as_stream(compute_stream);
  // one launch per step on the TMA path (float, stencil 2, unbatched)
  bool qpath = false;
  if constexpr (is_float<T>() && ST == 2) qpath = L.has_domain && QRun<true>::eligible(L.g, nt);
  QRun<true> qr;
  if constexpr (is_float<T>()) {
    float *const fl[3] = {lambda_ey, lambda_hx, lambda_hz};
    const float *const c3[3] = {ca, cb, cq};
    if (qpath && !qr.init(L.g, fl, c3, nullptr, nullptr, st)) return;
  }
  cudaStream_t ss = as_stream(storage_stream);
  const bool host_side = grads && (storage_mode == 1 || storage_mode == 2);
  const bool pipeline = host_side && ss != nullptr && ss != st;
  const size_t SN = (size_t)n_shots * (size_t)L.g.N;
  // disk mode: readers per snapshot kind into the host staging ring (*_store_3)
  std::unique_ptr<DiskHistory> disk[2];
  EventRing staged;  // the staging slot's host-to-device copy has completed
  if (grads && storage_mode == 2) {
    if (!staged.ok) {
      set_error(kCudaError, "TM2D: event creation failed");
      return;
    }
    const char *names[2] = {ca_requires_grad ? ey_filenames[0] : nullptr,
                            cb_requires_grad ? curl_filenames[0] : nullptr};
    for (int k = 0; k < 2; ++k)
      if (names[k]) {
        disk[k].reset(new DiskHistory(names[k], false, kRing));
        if (!disk[k]->ok()) {
          set_error(kBadArgument, "TM2D disk storage: %s", disk[k]->error().c_str());
          return;
        }
      }
  }
  bool staged_used[kRing] = {false, false, false};
  // Both ping-pong buffers of every CPML memory adjoint hold zeros outside
  // their strips for the whole call, so the kernels only write strip cells.
  if (TB_CUDA(cudaMemsetAsync(adjoint_memory_scratch, 0, 4 * SN * sizeof(T), st))) return;
  if (!zero_band(m_lambda_hz_x, L.g, 1, L.g.pml_x0, L.g.pml_x1, st) ||
      !zero_band(m_lambda_hx_z, L.g, 0, L.g.pml_y0, L.g.pml_y1, st) ||
      !zero_band(m_lambda_ey_x, L.g, 1, L.g.pml_x0, L.g.pml_x1h, st) ||
      !zero_band(m_lambda_ey_z, L.g, 0, L.g.pml_y0, L.g.pml_y1h, st))
    return;
  PointScratch ps;
  if (!build_points(ps, L, qpath ? qr.point_tiles() : L.ah_tiles(), sources_i,
                    n_sources_per_shot, receivers_i, n_receivers_per_shot, st))
    return;

  // Store indices consumed by this call, latest first.
  std::vector<int64_t> qs;
  if (grads)
    for (int64_t t = start_t - 1; t >= start_t - nt; --t)
      if (t % step_ratio == 0) qs.push_back(t / step_ratio);
  const size_t step_bytes = (size_t)shot_bytes_uncomp * (size_t)bg_shots;
  EventRing loaded, consumed;
  if (pipeline && (!loaded.ok || !consumed.ok)) {
    set_error(kCudaError, "TM2D: event creation failed");
    return;
  }
  if (pipeline)
    for (int k = 0; k < kRing; ++k)
      if (TB_CUDA(cudaEventRecord(consumed.ev[k], st))) return;
  // cpu storage mode: copy store index qs[n] from the pinned host history into
  // its device ring slot, on the side stream once the slot's last reader ran.
  auto load = [&](size_t n) -> bool {
    if (n >= qs.size()) return true;
    const int64_t q = qs[n];
    const int slot = (int)(q % kRing);
    cudaStream_t ls = pipeline ? ss : st;
    if (pipeline && TB_CUDA(cudaStreamWaitEvent(ss, consumed.ev[slot], 0))) return false;
    const bool from_disk = storage_mode == 2;
    const size_t off1 = (size_t)slot * step_bytes;
    const size_t off3 = from_disk ? (size_t)slot * step_bytes : (size_t)q * step_bytes;
    if (from_disk && staged_used[slot] && TB_CUDA(cudaEventSynchronize(staged.ev[slot])))
      return false;  // the staging slot's previous copy to the device has finished
    void *d1[2] = {ca_requires_grad ? (char *)ey_store_1 + off1 : nullptr,
                   cb_requires_grad ? (char *)curl_store_1 + off1 : nullptr};
    char *h3[2] = {(char *)ey_store_3 + off3, (char *)curl_store_3 + off3};
    for (int k = 0; k < 2; ++k) {
      if (!d1[k]) continue;
      if (from_disk && !disk[k]->read(h3[k], step_bytes, (int64_t)(q * step_bytes))) {
        set_error(kBadArgument, "TM2D disk storage: %s", disk[k]->error().c_str());
        return false;
      }
      if (TB_CUDA(cudaMemcpyAsync(d1[k], h3[k], step_bytes, cudaMemcpyHostToDevice, ls)))
        return false;
    }
    if (from_disk) {
      if (TB_CUDA(cudaEventRecord(staged.ev[slot], ls))) return false;
      staged_used[slot] = true;
    }
    if (pipeline && TB_CUDA(cudaEventRecord(loaded.ev[slot], ss))) return false;
    return true;
  };
  size_t next_q = 0;
  if (host_side)
    for (size_t n = 0; n < std::min<size_t>(2, qs.size()); ++n)
      if (!load(n)) return;

  T *cur_ey_x = m_lambda_ey_x, *cur_ey_z = m_lambda_ey_z;
  T *cur_hx_z = m_lambda_hx_z, *cur_hz_x = m_lambda_hz_x;
  T *nxt_ey_x = adjoint_memory_scratch, *nxt_ey_z = adjoint_memory_scratch + SN;
  T *nxt_hx_z = adjoint_memory_scratch + 2 * SN, *nxt_hz_x = adjoint_memory_scratch + 3 * SN;
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;

  ProfileScope prof(st);
  // One-sweep TMA steps.
  for (int64_t t = start_t - 1; qpath && t >= start_t - nt; --t) {
    if constexpr (is_float<T>()) {
      const bool smp = prof.sample(t);
      const bool grad_step = grads && t % step_ratio == 0;
      const int64_t q = t / step_ratio;
      const size_t off1 = storage_mode == 0 ? (size_t)q * step_bytes
                                            : (size_t)(q % kRing) * step_bytes;
      if (grad_step && pipeline &&
          TB_CUDA(cudaStreamWaitEvent(st, loaded.ev[(int)(q % kRing)], 0)))
        return;
      const char *es = grad_step && ca_requires_grad ? (const char *)ey_store_1 + off1 : nullptr;
      const char *cs = grad_step && cb_requires_grad ? (const char *)curl_store_1 + off1 : nullptr;
      const float *const mc[4] = {cur_hz_x, cur_hx_z, cur_ey_x, cur_ey_z};
      float *const mn[4] = {nxt_hz_x, nxt_hx_z, nxt_ey_x, nxt_ey_z};
      const float *grt = grad_r ? grad_r + t * rs : nullptr;
      float *gft = grad_f ? grad_f + t * fs : nullptr;
      if (smp) prof.begin(kKAdjStep);
      const bool ok =
          bf16 ? qr.template adj_step<__nv_bfloat16>(
                     L.g, ps, grt, gft, mc, mn, (const __nv_bfloat16 *)es,
                     (const __nv_bfloat16 *)cs, bg_shots, grad_ca, grad_cb, (float)step_ratio)
               : qr.template adj_step<float>(L.g, ps, grt, gft, mc, mn, (const float *)es,
                                             (const float *)cs, bg_shots, grad_ca, grad_cb,
                                             (float)step_ratio);
      if (!ok) return;
      if (smp) prof.end(kKAdjStep);
      std::swap(cur_hx_z, nxt_hx_z);
      std::swap(cur_hz_x, nxt_hz_x);
      std::swap(cur_ey_x, nxt_ey_x);
      std::swap(cur_ey_z, nxt_ey_z);
      if (grad_step && host_side) {
        ++next_q;
        if (pipeline && TB_CUDA(cudaEventRecord(consumed.ev[(int)(q % kRing)], st))) return;
        if (!load(next_q + 1)) return;
      }
    }
  }
  // Per-cell kernels; with the history on the device (or none) the step
  // blocks are replayed from a graph (run_step_blocks).
  const int64_t snap = grads ? (int64_t)(step_bytes / esz) : 0;
  // one snapshot per shot: the kernel indexes snapshots by shot directly
  // (GradArgs::snap_base skips its modulo)
  const int ga_bg = bg_shots == n_shots ? 0 : bg_shots;
  auto step = [&](int64_t i, cudaStream_t s, const int64_t *blk, int64_t B, bool smp) -> bool {
    const int64_t t = start_t - 1 - i;
    if (L.has_domain) {
      if (smp) prof.begin(kKAdjE);
      launch_adj_e<T, ST>(L, s, cb, lambda_ey, lambda_hx, lambda_hz, cur_hx_z, cur_hz_x,
                          nxt_hx_z, nxt_hz_x);
      if (smp) prof.end(kKAdjE);
    }
    std::swap(cur_hx_z, nxt_hx_z);
    std::swap(cur_hz_x, nxt_hz_x);
    const bool grad_step = grads && t % step_ratio == 0;
    const int64_t q = t / step_ratio;
    const size_t off1 = storage_mode == 0 ? (size_t)q * step_bytes
                                          : (size_t)(q % kRing) * step_bytes;
    if (grad_step && pipeline &&
        TB_CUDA(cudaStreamWaitEvent(s, loaded.ev[(int)(q % kRing)], 0)))
      return false;
    const char *es = grad_step && ca_requires_grad ? (const char *)ey_store_1 + off1 : nullptr;
    const char *cs = grad_step && cb_requires_grad ? (const char *)curl_store_1 + off1 : nullptr;
    const T *grt = grad_r ? grad_r + t * rs : nullptr;
    T *gft = grad_f ? grad_f + t * fs : nullptr;
    // the adjoint walks the steps backwards: pointers move down by a block
    const StepShift sh{blk, -B * fs, -B * rs, -(B / step_ratio) * snap};
    if (smp) prof.begin(kKAdjH);
    if (bf16) {
      GradArgs<T, __nv_bfloat16> ga{(const __nv_bfloat16 *)es, (const __nv_bfloat16 *)cs,
                                    grad_ca, grad_cb, (T)step_ratio, ca_batched, cb_batched,
                                    ga_bg};
      launch_adj_h<T, ST, __nv_bfloat16>(L, s, ca, cq, lambda_hx, lambda_hz, lambda_ey,
                                         cur_ey_x, cur_ey_z, nxt_ey_x, nxt_ey_z, ps, grt, gft,
                                         ga, sh);
    } else {
      GradArgs<T, T> ga{(const T *)es, (const T *)cs, grad_ca, grad_cb, (T)step_ratio,
                        ca_batched, cb_batched, ga_bg};
      launch_adj_h<T, ST, T>(L, s, ca, cq, lambda_hx, lambda_hz, lambda_ey, cur_ey_x,
                             cur_ey_z, nxt_ey_x, nxt_ey_z, ps, grt, gft, ga, sh);
    }
    if (smp) prof.end(kKAdjH);
    std::swap(cur_ey_x, nxt_ey_x);
    std::swap(cur_ey_z, nxt_ey_z);
    if (grad_step && host_side) {
      ++next_q;
      if (pipeline && TB_CUDA(cudaEventRecord(consumed.ev[(int)(q % kRing)], s))) return false;
      if (!load(next_q + 1)) return false;
    }
    return true;
  };
  if (!qpath) {
    if (host_side) {
      for (int64_t i = 0; i < nt; ++i)
        if (!step(i, st, nullptr, 0, prof.sample(start_t - 1 - i))) return;
    } else if (!run_step_blocks(nt, grads ? step_ratio : 1, st, prof, t_down, start_t, step)) {
      return;
    }
  }
  // Leave the final adjoint memories in the caller's arrays
  // (maxwell_tm_cuda_inst.cu:1256-1277).
  const size_t nbytes = SN * sizeof(T);
  if (cur_ey_x != m_lambda_ey_x) {
    if (TB_CUDA(cudaMemcpyAsync(m_lambda_ey_x, cur_ey_x, nbytes, cudaMemcpyDeviceToDevice, st)))
      return;
    if (TB_CUDA(cudaMemcpyAsync(m_lambda_ey_z, cur_ey_z, nbytes, cudaMemcpyDeviceToDevice, st)))
      return;
    if (TB_CUDA(cudaMemcpyAsync(m_lambda_hx_z, cur_hx_z, nbytes, cudaMemcpyDeviceToDevice, st)))
      return;
    if (TB_CUDA(cudaMemcpyAsync(m_lambda_hz_x, cur_hz_x, nbytes, cudaMemcpyDeviceToDevice, st)))
      return;
  }
  count_launches(qpath ? nt : nt * (L.has_domain ? 2 : 1));
  if (TB_CUDA(cudaGetLastError())) return;
  if constexpr (is_float<T>()) {
    if (qpath && !qr.finish()) return;
  }
  if (pipeline) TB_CUDA(cudaStreamSynchronize(ss));
  // disk mode: the staging ring is the caller's and is refilled by the next
  // call, so every copy out of it has finished before returning
  else if (grads && storage_mode == 2) TB_CUDA(cudaStreamSynchronize(st));
}

}  // namespace
}  // namespace tb

#define TB_DEFINE(S, T)                                                        \
  extern "C" void maxwell_tm_##S##_##T##_forward_cuda(TIDE_TM_FORWARD_ARGS(T)) { \
    tb::tm_forward<T, S>(                                                      \
        ca, cb, cq, f, ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x, debye_a, debye_b, debye_cp, \
        polarization, ey_prev, r, n_poles, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx,   \
        kxh, sources_i, receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx, n_sources_per_shot,   \
        n_receivers_per_shot, step_ratio, has_dispersion, ca_batched, cb_batched, cq_batched, \
        start_t, pml_y0, pml_x0, pml_y1, pml_x1, n_threads, device, compute_stream);          \
  }                                                                            \
  extern "C" void maxwell_tm_##S##_##T##_forward_with_storage_cuda(            \
      TIDE_TM_FORWARD_WITH_STORAGE_ARGS(T)) {                                  \
    tb::tm_forward_with_storage<T, S>(                                         \
        ca, cb, cq, f, ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x, r, ey_store_1, ey_store_3, \
        ey_filenames, curl_store_1, curl_store_3, curl_filenames, ay, by, ayh, byh, ax, bx,   \
        axh, bxh, ky, kyh, kx, kxh, sources_i, receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx, \
        n_sources_per_shot, n_receivers_per_shot, step_ratio, storage_mode, storage_format,   \
        shot_bytes_uncomp, ca_requires_grad, cb_requires_grad, ca_batched, cb_batched,        \
        cq_batched, start_t, pml_y0, pml_x0, pml_y1, pml_x1, n_threads, device,               \
        compute_stream, storage_stream);                                       \
  }                                                                            \
  extern "C" void maxwell_tm_##S##_##T##_backward_cuda(TIDE_TM_BACKWARD_ARGS(T)) { \
    tb::tm_backward<T, S>(                                                     \
        ca, cb, cq, grad_r, lambda_ey, lambda_hx, lambda_hz, m_lambda_ey_x, m_lambda_ey_z,    \
        m_lambda_hx_z, m_lambda_hz_x, adjoint_memory_scratch, ey_store_1, ey_store_3,         \
        ey_filenames, curl_store_1, curl_store_3, curl_filenames, grad_f, grad_ca, grad_cb,   \
        grad_ca_shot, grad_cb_shot, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh,     \
        sources_i, receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx, n_sources_per_shot,        \
        n_receivers_per_shot, step_ratio, storage_mode, storage_format, shot_bytes_uncomp,    \
        ca_requires_grad, cb_requires_grad, ca_batched, cb_batched, cq_batched, start_t,      \
        pml_y0, pml_x0, pml_y1, pml_x1, n_threads, device, compute_stream, storage_stream,    \
        n_shots);                                                              \
  }                                                                            \
  extern "C" void maxwell_tm_##S##_##T##_background_vjp_reuse_cuda(            \
      TIDE_TM_BACKGROUND_VJP_REUSE_ARGS(T)) {                                  \
    tb::tm_backward<T, S>(                                                     \
        ca, cb, cq, grad_r, lambda_ey, lambda_hx, lambda_hz, m_lambda_ey_x, m_lambda_ey_z,    \
        m_lambda_hx_z, m_lambda_hz_x, adjoint_memory_scratch, ey_store_1, ey_store_3,         \
        ey_filenames, curl_store_1, curl_store_3, curl_filenames, grad_f, grad_ca, grad_cb,   \
        grad_ca_shot, grad_cb_shot, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh,     \
        sources_i, receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx, n_sources_per_shot,        \
        n_receivers_per_shot, step_ratio, storage_mode, storage_format, shot_bytes_uncomp,    \
        ca_requires_grad, cb_requires_grad, ca_batched, cb_batched, cq_batched, start_t,      \
        pml_y0, pml_x0, pml_y1, pml_x1, n_threads, device, compute_stream, storage_stream,    \
        background_n_shots);                                                   \
  }

TB_DEFINE(2, float)
TB_DEFINE(4, float)
TB_DEFINE(6, float)
TB_DEFINE(8, float)
TB_DEFINE(2, double)
TB_DEFINE(4, double)
TB_DEFINE(6, double)
TB_DEFINE(8, double)

extern "C" int tide_b200_set_tma_ctas(int max_ctas) {
  return tb::g_tma_max_ctas.exchange(max_ctas < 0 ? 0 : max_ctas);
}

extern "C" int tide_b200_set_tma_mode(int mode) {
  return tb::g_tma_mode.exchange(mode < 0 ? 0 : (mode > 2 ? 2 : mode));
}
extern "C" int tide_b200_set_step_graphs(int on) { return tb::g_step_graphs.exchange(on ? 1 : 0); }
extern "C" int64_t tide_b200_graph_replays(void) { return tb::g_graph_replays.load(); }

extern "C" int64_t tide_b200_set_fused_threshold(int64_t bytes) {
  return tb::g_fused_min_bytes.exchange(bytes < 0 ? -1 : bytes);
}

extern "C" int tide_b200_device_status(int64_t device) {
  if (TB_CUDA(cudaSetDevice((int)device))) return -1;
  if (TB_CUDA(cudaDeviceSynchronize())) return -1;
  int v = 0;
  if (TB_CUDA(cudaMemcpyFromSymbol(&v, tb::g_tide_dev_err, sizeof(int)))) return -1;
  const int zero = 0;
  if (TB_CUDA(cudaMemcpyToSymbol(tb::g_tide_dev_err, &zero, sizeof(int)))) return -1;
  return v;
}

// ---------------------------------------------------------------------------
// Allocation-free forward (stencil 2, float).
//
// Some callers cannot allocate device memory while they run the solver: code
// executing inside a custom allocator or memory-pool callback, applications
// that reserve all device memory up front and forbid further allocation, and
// embedders whose own allocator is not the CUDA runtime's.  The regular
// forward allocates a small per-call scratch (the per-tile lists of source and
// receiver entries) from the stream-ordered pool; this variant instead keeps
// that scratch in one fixed device array that lives in this library, so the
// call performs no allocation and no free of any kind.
//
// Limits and sharing:
//  - the array holds kNoAllocScratchWords 32-bit words (16 MiB).  A call
//    needs 2 (tiles + 1) + 2 entries words per point list (sources and
//    receivers), tiles = n_shots * ceil(nx / 32) * ceil(ny / 16); larger
//    problems are rejected with a status message before any GPU work;
//  - every call on a device uses the same array and leaves its contents
//    behind; each call clears the counters it needs first.  Calls whose GPU
//    work overlaps (for example on two streams at once) race on the array and
//    must be serialised by the caller;
//  - every call looks the array's device address up with cudaGetSymbolAddress
//    (the device selected by `device` current), so the address stays valid
//    after a device reset reloads the module; the first call on a device may
//    load the library's device code, so make it before any stream capture.
namespace tb {
namespace {

constexpr size_t kNoAllocScratchWords = size_t(1) << 22;
static __device__ __align__(256) int g_noalloc_scratch[kNoAllocScratchWords];

// Device address of the scratch array on the current device.  Looked up on
// every call: cheap, allocates nothing, and never stale after a device reset.
int *noalloc_scratch() {
  void *p = nullptr;
  if (TB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch))) return nullptr;
  return static_cast<int *>(p);
}

}  // namespace
}  // namespace tb

extern "C" void maxwell_tm_2_float_forward_noalloc_cuda(TIDE_TM_FORWARD_ARGS(float)) {
  using namespace tb;
  using T = float;
  constexpr int ST = 2;
  (void)dt; (void)step_ratio; (void)n_threads; (void)ey_prev;
  (void)debye_a; (void)debye_b; (void)debye_cp; (void)polarization; (void)n_poles;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0, "noalloc forward: nt must be >= 0");
  TB_REQUIRE(!has_dispersion, "noalloc forward: Debye media are not supported by this variant");
  TB_REQUIRE(ca && cb && cq && ey && hx && hz && m_ey_x && m_ey_z && m_hx_z && m_hz_x,
             "noalloc forward: a field or coefficient pointer is null");
  TB_REQUIRE(n_sources_per_shot == 0 || f, "noalloc forward: sources without amplitudes");
  TB_REQUIRE(n_receivers_per_shot == 0 || r, "noalloc forward: receivers without output");
  Launch<T, ST> L;
  if (!make_launch(L, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, rdy, rdx, n_shots,
                   ny, nx, pml_y0, pml_x0, pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  const bool want_s = n_sources_per_shot > 0 && sources_i != nullptr;
  const bool want_r = n_receivers_per_shot > 0 && receivers_i != nullptr;
  const size_t nt1 = (size_t)L.tiles_x * L.tiles_y_e * (size_t)n_shots + 1;
  const size_t ns = want_s ? (size_t)(n_sources_per_shot * n_shots) : 0;
  const size_t nr = want_r ? (size_t)(n_receivers_per_shot * n_shots) : 0;
  const size_t words = (want_s ? 2 * nt1 + 2 * ns : 0) + (want_r ? 2 * nt1 + 2 * nr : 0);
  TB_REQUIRE(words <= kNoAllocScratchWords,
             "noalloc forward: problem needs %zu scratch words, the fixed array holds %zu "
             "(reduce n_shots per call or use maxwell_tm_2_float_forward_cuda)",
             words, kNoAllocScratchWords);
  int *scratch = noalloc_scratch();
  if (scratch == nullptr) return;
  cudaStream_t st = as_stream(compute_stream);
  PointScratch ps;  // ps.mem stays null: nothing is freed at scope exit
  ps.st = st;
  const int tile_h = kBlockY * kRowsE;
  int *w = scratch;
  if (want_s) {
    int *count = w, *start = w + nt1, *cell = w + 2 * nt1, *ent = w + 2 * nt1 + ns;
    if (!build_list(sources_i, (int)n_sources_per_shot, (int)n_shots, L.g.N, L.g.nx,
                    PointTiles{L.tiles_x, L.tiles_y_e, kTileX, tile_h, 0}, (int)(nt1 - 1), count,
                    start, cell, ent, st, ps.src))
      return;
    w += 2 * nt1 + 2 * ns;
  }
  if (want_r) {
    int *count = w, *start = w + nt1, *cell = w + 2 * nt1, *ent = w + 2 * nt1 + nr;
    if (!build_list(receivers_i, (int)n_receivers_per_shot, (int)n_shots, L.g.N, L.g.nx,
                    PointTiles{L.tiles_x, L.tiles_y_e, kTileX, tile_h, 0}, (int)(nt1 - 1), count,
                    start, cell, ent, st, ps.rec))
      return;
  }
  const DebyeArgs<T> db{nullptr, nullptr, nullptr, nullptr, 0};
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  for (int64_t t = start_t; t < start_t + nt; ++t) {
    if (L.has_domain) launch_fwd_h<T, ST>(L, st, cq, ey, hx, hz, m_ey_x, m_ey_z);
    launch_fwd_e<T, ST, T>(L, st, ca, cb, hx, hz, ey, m_hx_z, m_hz_x, nullptr, nullptr, db, ps,
                           f ? f + t * fs : nullptr, r ? r + t * rs : nullptr);
  }
  count_launches(nt * (L.has_domain ? 2 : 1));
  TB_CUDA(cudaGetLastError());
}

// Multi-job serving engine (shares this file's launch helpers and tile lists).
#include "tm2d_serve.cuh"

// Debye-medium forward with storage and adjoint (same launch helpers).
#include "tm2d_debye.cuh"

// Born (tangent) forward of the linearization (same launch helpers).
#include "tm2d_born.cuh"
