/* Multi-job TM2D serving engine of libtide_b200.so (stencil order 2, float32).
 *
 * The reference has no serving path: each tide.MaxwellTM call runs one job
 * (all of its shots) through the per-call entry points of tide_b200.h
 * (maxwell_tm_2_float_{forward,forward_with_storage,backward}_cuda, which
 * replace src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1281-1609).  This engine
 * advances many resident jobs of different grid shapes, shot counts and time
 * positions together: one launch per kernel kind and time step covers the
 * tiles of every job, so small jobs no longer pay a launch per kernel per
 * step each, and a forward-only job, a job recording snapshots and a job
 * running its adjoint share the device in the same step.  The per-cell
 * arithmetic is that of the per-call kernels (the same tile functions), so a
 * job's receivers, adjoint fields and gradients are bit-identical to the
 * per-call path whatever else is resident.  Large jobs run the per-call
 * kernels themselves on the engine's streams, next to the shared launches.
 *
 * Use: create an engine; bind each admitted job's device buffers to a slot
 * (bind builds the job's source/receiver tile lists once); before each chunk
 * plan every bound slot (phase, first step, number of steps, snapshot
 * buffers); run the chunk; release a slot when its job is done.  Every call
 * returns a status (0 ok, else see tide_b200_last_error); none exits the
 * process.  The engine works on its own streams and orders itself after /
 * before the caller's stream at each run.
 */
#ifndef TIDE_B200_SERVE_H
#define TIDE_B200_SERVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Device buffers and geometry of one job (all pointers are device pointers;
 * arrays are contiguous).  Geometry and profiles as in the per-call forward
 * (pml_* are the inner CPML edges, profiles are the 12 1-D arrays). */
typedef struct TideServeJob {
  int64_t n_shots, ny, nx, nt;
  int64_t pml_y0, pml_x0, pml_y1, pml_x1;
  double rdy, rdx;
  const float *ay, *by, *ayh, *byh, *ax, *bx, *axh, *bxh, *ky, *kyh, *kx, *kxh;
  const float *ca, *cb, *cq;                     /* [ny, nx] */
  float *ey, *hx, *hz, *m_ey_x, *m_ey_z, *m_hx_z, *m_hz_x; /* [S, ny, nx] */
  const float *f;                                /* [nt, S, n_src] (scaled amplitudes) */
  float *r;                                      /* [nt, S, n_rec] */
  const int64_t *sources_i, *receivers_i;        /* [S, n_src], [S, n_rec] flat cells */
  int64_t n_src, n_rec;
  /* Adjoint (null when the job is forward-only).  lam: lambda_ey, lambda_hx,
   * lambda_hz, then the memories of Ey-x, Ey-z, Hx-z, Hz-x; lam_scratch is
   * [4, S, ny, nx], the ping-pong partners of the four memories.  All must be
   * zero when the adjoint starts. */
  float *lam[7];
  float *lam_scratch;
  const float *grad_r;                           /* [nt, S, n_rec] */
  float *grad_f;                                 /* [nt, S, n_src] or null */
  float *grad_ca, *grad_cb;                      /* [ny, nx], accumulated into */
  int64_t step_ratio;                            /* gradient sampling interval k */
  int64_t storage_format;                        /* the engine's snapshot format */
} TideServeJob;

/* Plan flags. */
enum {
  /* the fields of this forward phase are not read after it (no checkpoint
   * copy, no later forward from them): a large slot may run it with the
   * fused pitched step */
  TIDE_SERVE_FLAG_FUSED = 1
};

/* Slot phases of a chunk. */
enum {
  TIDE_SERVE_IDLE = 0,
  TIDE_SERVE_FORWARD = 1,       /* steps t0 .. t0+n-1 */
  TIDE_SERVE_FORWARD_STORE = 2, /* same, recording snapshots at t % k == 0 */
  TIDE_SERVE_ADJOINT = 3        /* steps t0-1 down to t0-n (t0 = start_t) */
};

/* storage_format: snapshot type of every job of the engine (0 float32, 1 bf16). */
void *tide_b200_serve_create(int64_t device, int64_t max_slots, int64_t storage_format);
void tide_b200_serve_destroy(void *engine);
/* Binds a job to a free slot (its tile lists are built after the work already
 * on `stream`); returns the slot index (>= 0) or -1. */
int64_t tide_b200_serve_bind(void *engine, const TideServeJob *job, int64_t stream);
/* Frees the slot once the engine's enqueued work is done with it. */
int64_t tide_b200_serve_release(void *engine, int64_t slot);
/* Plans one slot for the next chunk.  Snapshot buffers (FORWARD_STORE and
 * ADJOINT; null for the other phases) hold store indices q0, q0+1, ... of
 * [S, ny, nx] steps each (store index q = t / k).  adj_parity is the number of
 * adjoint steps the job has already run (selects the current half of each
 * memory ping-pong pair). */
int64_t tide_b200_serve_plan(void *engine, int64_t slot, int64_t phase, int64_t t0,
                             int64_t n_steps, void *ey_store, void *curl_store, int64_t q0,
                             int64_t adj_parity, int64_t flags);
/* Runs chunk_steps steps of every planned slot (a slot with n_steps < chunk_steps
 * idles after its own steps).  use_graph != 0 replays a captured CUDA graph of
 * the chunk.  Ordered after the work already on `stream` and before later work
 * on it; returns once enqueued. */
int64_t tide_b200_serve_run(void *engine, int64_t chunk_steps, int64_t use_graph,
                            int64_t stream);
/* Slots of at least direct_cells shots x cells (bound after this call; < 0:
 * none) run the per-call kernels on their own streams instead of the shared
 * tile walk; fused != 0 lets them use the fused forward step when planned
 * with TIDE_SERVE_FLAG_FUSED.  Defaults: 1 << 20 cells, fused on. */
int64_t tide_b200_serve_configure(void *engine, int64_t direct_cells, int64_t fused);
/* Streams the large slots bound from now on are spread over (1..8; default
 * 8).  One stream runs the large slots of a chunk one after another, each
 * with its fields in L2 between its kernels; more streams overlap them.
 * Returns the previous count, or -1. */
int64_t tide_b200_serve_set_direct_streams(void *engine, int64_t n);
/* Kernel launches issued by the engine so far (graph replays count their nodes). */
int64_t tide_b200_serve_launches(void *engine);

#ifdef __cplusplus
}
#endif

#endif /* TIDE_B200_SERVE_H */
