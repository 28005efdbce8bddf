/*
 * tide_b200.h — C ABI of libtide_b200.so, the B200 (sm_100a) implementation
 * of TIDE's native time-stepping paths: 2-D TM and 3-D Maxwell (Yee).
 *
 * The exported symbols carry the reference backend's names and argument
 * lists, so the reference's ctypes loader can bind them unchanged:
 *   symbol naming   src/tide/backend_utils.py:771-787
 *                   ("{propagator}_{accuracy}_{dtype}_{pass}_{device}")
 *   argument specs  src/tide/backend_utils.py:227-308 (TM forward,
 *                   forward_with_storage, backward), :446-556 (3-D)
 * Every pointer is a raw device (or pinned host, where stated) address; sizes
 * are int64; no torch types cross this boundary.
 *
 * Differences from the reference behaviour (all deliberate):
 *   - No entry point ever exits or aborts the process.  A failed argument
 *     check or CUDA call records a status readable through
 *     tide_b200_last_error() and the call returns early.
 *   - Geometry travels as kernel arguments, never as process-global
 *     __constant__ state, so concurrent calls with different shapes on
 *     different streams are safe.
 *   - backward clears the per-shot accumulators on entry and writes batched
 *     model gradients straight into grad_ca/grad_cb, as the reference CPU
 *     backend does (maxwell_tm_inst.cpp:2050-2206).
 */
#ifndef TIDE_B200_H
#define TIDE_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Argument list of maxwell_tm_*_forward_cuda.  Replaces
 * maxwell_tm_{S}_{dtype}_forward_cuda, src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1281-1368
 * (argtypes src/tide/backend_utils.py:256-269). */
#define TIDE_TM_FORWARD_ARGS(T)                                                \
  T const *ca, T const *cb, T const *cq, T const *f, T *ey, T *hx, T *hz,      \
      T *m_ey_x, T *m_ey_z, T *m_hx_z, T *m_hz_x, T const *debye_a,            \
      T const *debye_b, T const *debye_cp, T *polarization, T *ey_prev, T *r,  \
      int64_t n_poles, T const *ay, T const *by, T const *ayh, T const *byh,  \
      T const *ax, T const *bx, T const *axh, T const *bxh, T const *ky,       \
      T const *kyh, T const *kx, T const *kxh, int64_t const *sources_i,       \
      int64_t const *receivers_i, T rdy, T rdx, T dt, int64_t nt,              \
      int64_t n_shots, int64_t ny, int64_t nx, int64_t n_sources_per_shot,     \
      int64_t n_receivers_per_shot, int64_t step_ratio, bool has_dispersion,   \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_y0, int64_t pml_x0, int64_t pml_y1, int64_t pml_x1,          \
      int64_t n_threads, int64_t device, void *compute_stream

/* Argument list of maxwell_tm_*_forward_with_storage_cuda.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1371-1609
 * (argtypes src/tide/backend_utils.py:271-287).  step_ratio is the gradient
 * sampling interval k: Ey^t and curl H^t are stored when t % k == 0.
 * storage_mode: 0 device, 1 cpu (pinned host history, 3-slot device ring),
 * 2 disk (3-slot device ring, 3-slot pinned staging ring passed as
 * *_store_3, the history in the file named by *_filenames[0]: stored step q
 * at byte offset q * n_shots * shot_bytes_uncomp, written by a background
 * thread; the call returns after its writes are on disk), 3 none.
 * storage_format: 0 full, 1 bf16. */
#define TIDE_TM_FORWARD_WITH_STORAGE_ARGS(T)                                   \
  T const *ca, T const *cb, T const *cq, T const *f, T *ey, T *hx, T *hz,      \
      T *m_ey_x, T *m_ey_z, T *m_hx_z, T *m_hz_x, T *r, void *ey_store_1,      \
      void *ey_store_3, char const *const *ey_filenames, void *curl_store_1,   \
      void *curl_store_3, char const *const *curl_filenames, T const *ay,      \
      T const *by, T const *ayh, T const *byh, T const *ax, T const *bx,       \
      T const *axh, T const *bxh, T const *ky, T const *kyh, T const *kx,      \
      T const *kxh, int64_t const *sources_i, int64_t const *receivers_i,      \
      T rdy, T rdx, T dt, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx, \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_y0, int64_t pml_x0, int64_t pml_y1, int64_t pml_x1,          \
      int64_t n_threads, int64_t device, void *compute_stream,                 \
      void *storage_stream

/* Argument list of maxwell_tm_*_backward_cuda.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:2739-2770 (which delegates to
 * background_vjp_reuse, :2405-2734); argtypes src/tide/backend_utils.py:289-308.
 * Runs t = start_t-1 down to start_t-nt. */
#define TIDE_TM_BACKWARD_ARGS(T)                                               \
  T const *ca, T const *cb, T const *cq, T const *grad_r, T *lambda_ey,        \
      T *lambda_hx, T *lambda_hz, T *m_lambda_ey_x, T *m_lambda_ey_z,          \
      T *m_lambda_hx_z, T *m_lambda_hz_x, T *adjoint_memory_scratch,           \
      void *ey_store_1, void *ey_store_3, char const *const *ey_filenames,     \
      void *curl_store_1, void *curl_store_3,                                  \
      char const *const *curl_filenames, T *grad_f, T *grad_ca, T *grad_cb,    \
      T *grad_ca_shot, T *grad_cb_shot, T const *ay, T const *by,              \
      T const *ayh, T const *byh, T const *ax, T const *bx, T const *axh,      \
      T const *bxh, T const *ky, T const *kyh, T const *kx, T const *kxh,      \
      int64_t const *sources_i, int64_t const *receivers_i, T rdy, T rdx,      \
      T dt, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx,               \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_y0, int64_t pml_x0, int64_t pml_y1, int64_t pml_x1,          \
      int64_t n_threads, int64_t device, void *compute_stream,                 \
      void *storage_stream

/* Argument list of maxwell_tm_*_background_vjp_reuse_cuda: the backward's,
 * with background_n_shots after shot_bytes_uncomp.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:2405-2460 (argtypes
 * src/tide/backend_utils.py:310-334; called by the Born autograd,
 * src/tide/maxwell/tm2d_born_autograd.py:886-960): the snapshot history holds
 * background_n_shots shots (n_shots must be a multiple of it) and adjoint
 * shot s images against snapshot shot s % background_n_shots. */
#define TIDE_TM_BACKGROUND_VJP_REUSE_ARGS(T)                                   \
  T const *ca, T const *cb, T const *cq, T const *grad_r, T *lambda_ey,        \
      T *lambda_hx, T *lambda_hz, T *m_lambda_ey_x, T *m_lambda_ey_z,          \
      T *m_lambda_hx_z, T *m_lambda_hz_x, T *adjoint_memory_scratch,           \
      void *ey_store_1, void *ey_store_3, char const *const *ey_filenames,     \
      void *curl_store_1, void *curl_store_3,                                  \
      char const *const *curl_filenames, T *grad_f, T *grad_ca, T *grad_cb,    \
      T *grad_ca_shot, T *grad_cb_shot, T const *ay, T const *by,              \
      T const *ayh, T const *byh, T const *ax, T const *bx, T const *axh,      \
      T const *bxh, T const *ky, T const *kyh, T const *kx, T const *kxh,      \
      int64_t const *sources_i, int64_t const *receivers_i, T rdy, T rdx,      \
      T dt, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx,               \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, int64_t background_n_shots,                   \
      bool ca_requires_grad, bool cb_requires_grad, bool ca_batched,           \
      bool cb_batched, bool cq_batched, int64_t start_t, int64_t pml_y0,       \
      int64_t pml_x0, int64_t pml_y1, int64_t pml_x1, int64_t n_threads,       \
      int64_t device, void *compute_stream, void *storage_stream

#define TIDE_TM_DECLARE(S, T)                                                  \
  void maxwell_tm_##S##_##T##_forward_cuda(TIDE_TM_FORWARD_ARGS(T));           \
  void maxwell_tm_##S##_##T##_forward_with_storage_cuda(                       \
      TIDE_TM_FORWARD_WITH_STORAGE_ARGS(T));                                   \
  void maxwell_tm_##S##_##T##_backward_cuda(TIDE_TM_BACKWARD_ARGS(T));         \
  void maxwell_tm_##S##_##T##_background_vjp_reuse_cuda(                       \
      TIDE_TM_BACKGROUND_VJP_REUSE_ARGS(T));

/* Stencil orders 2/4/6/8 in float and double, as the reference exports
 * (src/tide/csrc/tm2d/maxwell_tm_cuda_instantiations.inc). */
TIDE_TM_DECLARE(2, float)
TIDE_TM_DECLARE(4, float)
TIDE_TM_DECLARE(6, float)
TIDE_TM_DECLARE(8, float)
TIDE_TM_DECLARE(2, double)
TIDE_TM_DECLARE(4, double)
TIDE_TM_DECLARE(6, double)
TIDE_TM_DECLARE(8, double)

/* Argument list of maxwell_tm_*_born_forward_cuda, the Born (tangent)
 * propagation behind operator.linearize(...).jvp.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1611-1703 (argtypes
 * src/tide/backend_utils.py:336-349).  Advances the background state (ey ..
 * m_hz_x, sources f0) and the scattered state (dey .. dm_hz_x, sources df)
 * together; the scattered E update adds dca Ey^n + dcb curl H^n of the
 * background.  r records the scattered Ey, background_r (may be null) the
 * background Ey, at the receivers.  dca/dcb follow ca_batched/cb_batched. */
#define TIDE_TM_BORN_FORWARD_ARGS(T)                                           \
  T const *ca, T const *cb, T const *cq, T const *dca, T const *dcb,           \
      T const *f0, T const *df, T *ey, T *hx, T *hz, T *m_ey_x, T *m_ey_z,     \
      T *m_hx_z, T *m_hz_x, T *dey, T *dhx, T *dhz, T *dm_ey_x, T *dm_ey_z,    \
      T *dm_hx_z, T *dm_hz_x, T *r, T *background_r, T const *ay,              \
      T const *by, T const *ayh, T const *byh, T const *ax, T const *bx,       \
      T const *axh, T const *bxh, T const *ky, T const *kyh, T const *kx,      \
      T const *kxh, int64_t const *sources_i, int64_t const *receivers_i,      \
      T rdy, T rdx, T dt, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx, \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, bool ca_batched, bool cb_batched, bool cq_batched,   \
      int64_t start_t, int64_t pml_y0, int64_t pml_x0, int64_t pml_y1,         \
      int64_t pml_x1, int64_t n_threads, int64_t device, void *compute_stream

/* maxwell_tm_*_born_forward_with_storage_cuda.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1701-2086 (argtypes
 * src/tide/backend_utils.py:351-370).  The Born
 * forward that also stores the background history the adjoint needs: Ey^n
 * (ca_requires_grad) and the CPML-corrected curl H^n (cb_requires_grad) at
 * steps t % step_ratio == 0, in the storage modes and formats of
 * forward_with_storage.  dey_store / dcurl_store (may be null) receive the
 * scattered dEy^n and dcurl H^n of the same steps in a device history
 * [n_store, n_shots, ny, nx] of the snapshot type. */
#define TIDE_TM_BORN_FORWARD_WITH_STORAGE_ARGS(T)                              \
  T const *ca, T const *cb, T const *cq, T const *dca, T const *dcb,           \
      T const *f0, T const *df, T *ey, T *hx, T *hz, T *m_ey_x, T *m_ey_z,     \
      T *m_hx_z, T *m_hz_x, T *dey, T *dhx, T *dhz, T *dm_ey_x, T *dm_ey_z,    \
      T *dm_hx_z, T *dm_hz_x, T *r, T *background_r, void *ey_store_1,         \
      void *ey_store_3, char const *const *ey_filenames, void *curl_store_1,   \
      void *curl_store_3, char const *const *curl_filenames, void *dey_store,  \
      void *dcurl_store, T const *ay, T const *by, T const *ayh, T const *byh, \
      T const *ax, T const *bx, T const *axh, T const *bxh, T const *ky,       \
      T const *kyh, T const *kx, T const *kxh, int64_t const *sources_i,       \
      int64_t const *receivers_i, T rdy, T rdx, T dt, int64_t nt,              \
      int64_t n_shots, int64_t ny, int64_t nx, int64_t n_sources_per_shot,     \
      int64_t n_receivers_per_shot, int64_t step_ratio, int64_t storage_mode,  \
      int64_t storage_format, int64_t shot_bytes_uncomp,                       \
      bool ca_requires_grad, bool cb_requires_grad, bool ca_batched,           \
      bool cb_batched, bool cq_batched, int64_t start_t, int64_t pml_y0,       \
      int64_t pml_x0, int64_t pml_y1, int64_t pml_x1, int64_t n_threads,       \
      int64_t device, void *compute_stream, void *storage_stream

/* maxwell_tm_*_born_backward_cuda.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:2088-2400 (argtypes
 * src/tide/backend_utils.py:386-405).  The adjoint of the
 * Born map for (dca, dcb, df): the scattered E update adds dca Ey^n + dcb
 * curl H^n of the background, so grad_ca / grad_cb are the background
 * history correlated with the adjoint Ey, exactly as in backward, and
 * grad_f is the adjoint at the sources.  The arguments are backward's
 * without adjoint_memory_scratch (the call allocates its CPML adjoint
 * ping-pong buffers in stream order) and with work_x / work_z (unused, as
 * in the reference). */
#define TIDE_TM_BORN_BACKWARD_ARGS(T)                                          \
  T const *ca, T const *cb, T const *cq, T const *grad_r, T *lambda_ey,        \
      T *lambda_hx, T *lambda_hz, T *m_lambda_ey_x, T *m_lambda_ey_z,          \
      T *m_lambda_hx_z, T *m_lambda_hz_x, void *ey_store_1, void *ey_store_3,  \
      char const *const *ey_filenames, void *curl_store_1, void *curl_store_3, \
      char const *const *curl_filenames, T *grad_f, T *grad_ca, T *grad_cb,    \
      T *grad_ca_shot, T *grad_cb_shot, T *work_x, T *work_z, T const *ay,     \
      T const *by, T const *ayh, T const *byh, T const *ax, T const *bx,       \
      T const *axh, T const *bxh, T const *ky, T const *kyh, T const *kx,      \
      T const *kxh, int64_t const *sources_i, int64_t const *receivers_i,      \
      T rdy, T rdx, T dt, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx, \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_y0, int64_t pml_x0, int64_t pml_y1, int64_t pml_x1,          \
      int64_t n_threads, int64_t device, void *compute_stream,                 \
      void *storage_stream

/* maxwell_tm_*_born_backward_bggrad_cuda.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:2785-3200 (argtypes
 * src/tide/backend_utils.py:407-440): the derivative of grad_r . (scattered
 * receivers) + grad_background_r . (background receivers) in the background
 * coefficients (grad_ca, grad_cb), the perturbation (grad_dca, grad_dcb) and
 * the background and scattered sources (grad_f0, grad_df), by the exact
 * adjoint of the joint background + scattered recurrence over the background
 * history (ey_store_1 / curl_store_1, [n_store, background_n_shots, ny, nx])
 * and the scattered history (dey_store / dcurl_store, [n_store, n_shots,
 * ny, nx]) of born_forward_with_storage, device storage mode.  ey / hx / hz
 * receive the scattered state's adjoint, dey / dhx / dhz the background's,
 * the eight memories theirs (all zeroed on entry); adjoint_memory_scratch
 * holds 8 n_shots ny nx values and work_eta_x n_shots ny nx; the gradients
 * accumulate, shot sums in-kernel (grad_*_shot, eta_source_old, work_eta_z
 * and lambda_store are not used).  capture_background_adjoint /
 * reuse_background_adjoint are rejected with a status message. */
#define TIDE_TM_BORN_BACKWARD_BGGRAD_ARGS(T)                                   \
  T const *ca, T const *cb, T const *cq, T const *dca, T const *dcb,           \
      T const *f0, T const *df, T const *grad_r, T const *grad_background_r,   \
      void *ey_store_1, void *ey_store_3, char const *const *ey_filenames,     \
      void *curl_store_1, void *curl_store_3, char const *const *curl_filenames, \
      void const *dey_store, void const *dcurl_store, void *lambda_store,      \
      int64_t background_n_shots, T *ey, T *hx, T *hz, T *dey, T *dhx, T *dhz, \
      T *grad_f0, T *grad_df, T *grad_ca, T *grad_cb, T *grad_dca, T *grad_dcb, \
      T *m_lambda_ey_x, T *m_lambda_ey_z, T *m_lambda_hx_z, T *m_lambda_hz_x,  \
      T *m_eta_ey_x, T *m_eta_ey_z, T *m_eta_hx_z, T *m_eta_hz_x,              \
      T *eta_source_old, T *work_eta_x, T *work_eta_z, T *grad_ca_shot,        \
      T *grad_cb_shot, T *grad_dca_shot, T *grad_dcb_shot,                     \
      T *adjoint_memory_scratch, T const *ay, T const *by, T const *ayh,       \
      T const *byh, T const *ax, T const *bx, T const *axh, T const *bxh,      \
      T const *ky, T const *kyh, T const *kx, T const *kxh,                    \
      int64_t const *sources_i, int64_t const *receivers_i, T rdy, T rdx,      \
      T dt, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx,               \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool capture_background_adjoint, bool reuse_background_adjoint,          \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_y0, int64_t pml_x0, int64_t pml_y1, int64_t pml_x1,          \
      int64_t n_threads, int64_t device, void *compute_stream,                 \
      void *storage_stream

/* maxwell_tm_*_born_tangent_forward_with_storage_cuda.  Replaces
 * src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1974-2086 (argtypes
 * src/tide/backend_utils.py:372-384).  Advances only the scattered state,
 * reading the background Ey^n / curl H^n of each step from a stored device
 * history [nt, background_n_shots, ny, nx] (snapshot type of
 * storage_format) instead of recomputing the background; scattered shot s
 * uses background shot s % background_n_shots (direction batches).
 * step_ratio must be 1.  r records the scattered Ey; dey_store /
 * dcurl_store (may be null) receive the scattered history
 * [nt, n_shots, ny, nx]. */
#define TIDE_TM_BORN_TANGENT_ARGS(T)                                           \
  T const *ca, T const *cb, T const *cq, T const *dca, T const *dcb,           \
      T const *df, T *dey, T *dhx, T *dhz, T *dm_ey_x, T *dm_ey_z,             \
      T *dm_hx_z, T *dm_hz_x, T *r, void const *ey_store,                      \
      void const *curl_store, void *dey_store, void *dcurl_store, T const *ay, \
      T const *by, T const *ayh, T const *byh, T const *ax, T const *bx,       \
      T const *axh, T const *bxh, T const *ky, T const *kyh, T const *kx,      \
      T const *kxh, int64_t const *sources_i, int64_t const *receivers_i,      \
      T rdy, T rdx, T dt, int64_t nt, int64_t n_shots, int64_t ny, int64_t nx, \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_format, int64_t background_n_shots,  \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_y0, int64_t pml_x0, int64_t pml_y1, int64_t pml_x1,          \
      int64_t n_threads, int64_t device, void *compute_stream

#define TIDE_TM_BORN_DECLARE(S, T)                                             \
  void maxwell_tm_##S##_##T##_born_forward_cuda(TIDE_TM_BORN_FORWARD_ARGS(T)); \
  void maxwell_tm_##S##_##T##_born_forward_with_storage_cuda(                  \
      TIDE_TM_BORN_FORWARD_WITH_STORAGE_ARGS(T));                              \
  void maxwell_tm_##S##_##T##_born_tangent_forward_with_storage_cuda(          \
      TIDE_TM_BORN_TANGENT_ARGS(T));                                           \
  void maxwell_tm_##S##_##T##_born_backward_cuda(TIDE_TM_BORN_BACKWARD_ARGS(T));        \
  void maxwell_tm_##S##_##T##_born_backward_bggrad_cuda(                       \
      TIDE_TM_BORN_BACKWARD_BGGRAD_ARGS(T));

TIDE_TM_BORN_DECLARE(2, float)
TIDE_TM_BORN_DECLARE(4, float)
TIDE_TM_BORN_DECLARE(6, float)
TIDE_TM_BORN_DECLARE(8, float)
TIDE_TM_BORN_DECLARE(2, double)
TIDE_TM_BORN_DECLARE(4, double)
TIDE_TM_BORN_DECLARE(6, double)
TIDE_TM_BORN_DECLARE(8, double)

/* Allocation-free variant of maxwell_tm_2_float_forward_cuda (same arguments,
 * same results).  It has no counterpart in the reference.  It is for callers
 * that must not allocate device memory during the call -- code running inside
 * an allocator or memory-pool callback, or applications that reserve all
 * device memory up front: the per-call scratch (the per-tile lists of source
 * and receiver entries) lives in a fixed 16 MiB device array inside this
 * library instead of the stream-ordered pool.  Problems needing more scratch
 * than the array holds (2 (tiles + 1) + 2 entries words per point list,
 * tiles = n_shots * ceil(nx/32) * ceil(ny/16)) are rejected with a status
 * message.  All calls on a device share the array, so calls whose GPU work
 * overlaps race and must be serialised.  Every call looks the array's
 * address up on the current device (nothing is cached, so a device reset is
 * harmless); the first call on a device may load the library's device code
 * and should come before any stream capture.  Debye
 * media are not supported by this variant. */
void maxwell_tm_2_float_forward_noalloc_cuda(TIDE_TM_FORWARD_ARGS(float));

/* ---------------------------------------------------------------- 3-D */

/* Argument list of maxwell_3d_*_forward_cuda.  Replaces
 * maxwell_3d_{S}_{dtype}_forward_cuda, src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:3012-3288
 * (argtypes src/tide/backend_utils.py:484-504).  Fields [S, nz, ny, nx];
 * CPML memories compacted along their own axis as the reference's CUDA
 * callers allocate them (grid_utils.py:96-150): axis extent
 * pml_0 + n - max(pml_0, pml_1 - 1).  source/receiver_component 0 x, 1 y, 2 z.
 * Dispersion (has_dispersion) and execution_backend != 0 are rejected with a
 * status message. */
#define TIDE_3D_FORWARD_ARGS(T)                                                \
  T const *ca, T const *cb, T const *cq, T const *f, T *ex, T *ey, T *ez,      \
      T *hx, T *hy, T *hz, T *m_hz_y, T *m_hy_z, T *m_hx_z, T *m_hz_x,         \
      T *m_hy_x, T *m_hx_y, T *m_ey_z, T *m_ez_y, T *m_ez_x, T *m_ex_z,        \
      T *m_ex_y, T *m_ey_x, T const *debye_a, T const *debye_b,                \
      T const *debye_cp, T *pol_ex, T *pol_ey, T *pol_ez, T *ex_prev,          \
      T *ey_prev, T *ez_prev, T *r, int64_t n_poles, T const *az, T const *bz, \
      T const *azh, T const *bzh, T const *ay, T const *by, T const *ayh,      \
      T const *byh, T const *ax, T const *bx, T const *axh, T const *bxh,      \
      T const *kz, T const *kzh, T const *ky, T const *kyh, T const *kx,       \
      T const *kxh, int64_t const *sources_i, int64_t const *receivers_i,      \
      T rdz, T rdy, T rdx, T dt, int64_t nt, int64_t n_shots, int64_t nz,      \
      int64_t ny, int64_t nx, int64_t n_sources_per_shot,                      \
      int64_t n_receivers_per_shot, int64_t step_ratio, bool has_dispersion,   \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_z0, int64_t pml_y0, int64_t pml_x0, int64_t pml_z1,          \
      int64_t pml_y1, int64_t pml_x1, int64_t source_component,                \
      int64_t receiver_component, int64_t n_threads, int64_t device,           \
      int64_t execution_backend, void *compute_stream

/* maxwell_3d_*_forward_with_storage_cuda.  Replaces
 * src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:3290-3880 (argtypes
 * src/tide/backend_utils.py:506-524).  Stores E^t (3 components) and the
 * CPML-corrected curl H (3 components) at steps t % step_ratio == 0; each
 * component has a device buffer (s1), a pinned host history (s3, cpu mode)
 * and a file-name list (fn, disk mode: one file name, char **). */
#define TIDE_3D_FORWARD_WITH_STORAGE_ARGS(T)                                   \
  T const *ca, T const *cb, T const *cq, T const *f, T *ex, T *ey, T *ez,      \
      T *hx, T *hy, T *hz, T *m_hz_y, T *m_hy_z, T *m_hx_z, T *m_hz_x,         \
      T *m_hy_x, T *m_hx_y, T *m_ey_z, T *m_ez_y, T *m_ez_x, T *m_ex_z,        \
      T *m_ex_y, T *m_ey_x, T *r, void *ex_s1, void *ex_s3, void *ex_fn,       \
      void *ey_s1, void *ey_s3, void *ey_fn, void *ez_s1, void *ez_s3,         \
      void *ez_fn, void *cx_s1, void *cx_s3, void *cx_fn, void *cy_s1,         \
      void *cy_s3, void *cy_fn, void *cz_s1, void *cz_s3, void *cz_fn,         \
      T const *az, T const *bz, T const *azh, T const *bzh, T const *ay,       \
      T const *by, T const *ayh, T const *byh, T const *ax, T const *bx,       \
      T const *axh, T const *bxh, T const *kz, T const *kzh, T const *ky,      \
      T const *kyh, T const *kx, T const *kxh, int64_t const *sources_i,       \
      int64_t const *receivers_i, T rdz, T rdy, T rdx, T dt, int64_t nt,       \
      int64_t n_shots, int64_t nz, int64_t ny, int64_t nx,                     \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_z0, int64_t pml_y0, int64_t pml_x0, int64_t pml_z1,          \
      int64_t pml_y1, int64_t pml_x1, int64_t source_component,                \
      int64_t receiver_component, int64_t n_threads, int64_t device,           \
      int64_t execution_backend, void *compute_stream, void *storage_stream

/* maxwell_3d_*_backward_cuda.  Replaces
 * src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:4542-5240 (argtypes
 * src/tide/backend_utils.py:537-556).  Exact adjoint over t = start_t-1 down
 * to start_t-nt; adjoint CPML memories ping-pong with adjoint_memory_scratch
 * (same compact sizes, the final state lands in the caller's arrays).
 * grad_ca / grad_cb accumulate; with several unbatched shots the per-shot
 * sums go to grad_*_shot and are added once at the end in shot order (then
 * cleared); grad_eps / grad_sigma, when given, receive the conversion of the
 * final grad_ca / grad_cb (maxwell_3d_cuda_inst.cu:2729-2776). */
#define TIDE_3D_BACKWARD_ARGS(T)                                               \
  T const *ca, T const *cb, T const *cq, T const *grad_r, T *lambda_ex,        \
      T *lambda_ey, T *lambda_ez, T *lambda_hx, T *lambda_hy, T *lambda_hz,    \
      T *m_lambda_ey_z, T *m_lambda_ez_y, T *m_lambda_ez_x, T *m_lambda_ex_z,  \
      T *m_lambda_ex_y, T *m_lambda_ey_x, T *m_lambda_hz_y, T *m_lambda_hy_z,  \
      T *m_lambda_hx_z, T *m_lambda_hz_x, T *m_lambda_hy_x, T *m_lambda_hx_y,  \
      T *adjoint_memory_scratch, void *ex_s1, void *ex_s3, void *ex_fn,        \
      void *ey_s1, void *ey_s3, void *ey_fn, void *ez_s1, void *ez_s3,         \
      void *ez_fn, void *cx_s1, void *cx_s3, void *cx_fn, void *cy_s1,         \
      void *cy_s3, void *cy_fn, void *cz_s1, void *cz_s3, void *cz_fn,         \
      T *grad_f, T *grad_ca, T *grad_cb, T *grad_eps, T *grad_sigma,           \
      T *grad_ca_shot, T *grad_cb_shot, bool zero_grad_on_entry, T const *az,  \
      T const *bz, T const *azh, T const *bzh, T const *ay, T const *by,       \
      T const *ayh, T const *byh, T const *ax, T const *bx, T const *axh,      \
      T const *bxh, T const *kz, T const *kzh, T const *ky, T const *kyh,      \
      T const *kx, T const *kxh, int64_t const *sources_i,                     \
      int64_t const *receivers_i, T rdz, T rdy, T rdx, T dt, int64_t nt,       \
      int64_t n_shots, int64_t nz, int64_t ny, int64_t nx,                     \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_z0, int64_t pml_y0, int64_t pml_x0, int64_t pml_z1,          \
      int64_t pml_y1, int64_t pml_x1, int64_t source_component,                \
      int64_t receiver_component, int64_t n_threads, int64_t device,           \
      int64_t execution_backend, void *compute_stream, void *storage_stream

#define TIDE_3D_DECLARE(S, T)                                                  \
  void maxwell_3d_##S##_##T##_forward_cuda(TIDE_3D_FORWARD_ARGS(T));           \
  void maxwell_3d_##S##_##T##_forward_with_storage_cuda(                       \
      TIDE_3D_FORWARD_WITH_STORAGE_ARGS(T));                                   \
  void maxwell_3d_##S##_##T##_backward_cuda(TIDE_3D_BACKWARD_ARGS(T));

/* Stencil orders 2, 4, 6, 8 (S): the update domain is [S/2, n - S/2 + 1)
 * per axis, with the model padded by S/2 cells before and S/2 - 1 after it
 * (maxwell3d_cuda.py:314-326). */
TIDE_3D_DECLARE(2, float)
TIDE_3D_DECLARE(2, double)
TIDE_3D_DECLARE(4, float)
TIDE_3D_DECLARE(4, double)
TIDE_3D_DECLARE(6, float)
TIDE_3D_DECLARE(6, double)
TIDE_3D_DECLARE(8, float)
TIDE_3D_DECLARE(8, double)

/* maxwell_3d_*_born_forward_cuda, the 3-D Born (tangent) propagation.
 * Replaces maxwell_3d_{S}_{dtype}_born_forward_cuda (CPU counterpart
 * src/tide/csrc/em3d/maxwell_3d_inst.cpp:1100-1527; argtypes
 * src/tide/backend_utils.py:556-577).  Background state (ex .. m_ey_x,
 * sources f0) and scattered state (dex .. dm_ey_x, sources df) advance
 * together; the scattered E update adds dca E^n + dcb curl H^n of the
 * background.  r records the scattered, background_r (may be null) the
 * background receiver component.  CPML memories are full [S, nz, ny, nx]
 * arrays on the Born entry points (the reference's Born callers allocate
 * them so; its forward / backward entry points use the compact layout). */
#define TIDE_3D_BORN_FORWARD_ARGS(T)                                           \
  T const *ca, T const *cb, T const *cq, T const *dca, T const *dcb,           \
      T const *f0, T const *df, T *ex, T *ey, T *ez, T *hx, T *hy, T *hz,      \
      T *m_hz_y, T *m_hy_z, T *m_hx_z, T *m_hz_x, T *m_hy_x, T *m_hx_y,        \
      T *m_ey_z, T *m_ez_y, T *m_ez_x, T *m_ex_z, T *m_ex_y, T *m_ey_x,        \
      T *dex, T *dey, T *dez, T *dhx, T *dhy, T *dhz, T *dm_hz_y, T *dm_hy_z,  \
      T *dm_hx_z, T *dm_hz_x, T *dm_hy_x, T *dm_hx_y, T *dm_ey_z, T *dm_ez_y,  \
      T *dm_ez_x, T *dm_ex_z, T *dm_ex_y, T *dm_ey_x, T *r, T *background_r,   \
      T const *az, T const *bz, T const *azh, T const *bzh, T const *ay,       \
      T const *by, T const *ayh, T const *byh, T const *ax, T const *bx,       \
      T const *axh, T const *bxh, T const *kz, T const *kzh, T const *ky,      \
      T const *kyh, T const *kx, T const *kxh, int64_t const *sources_i,       \
      int64_t const *receivers_i, T rdz, T rdy, T rdx, T dt, int64_t nt,       \
      int64_t n_shots, int64_t nz, int64_t ny, int64_t nx,                     \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, bool ca_batched, bool cb_batched, bool cq_batched,   \
      int64_t start_t, int64_t pml_z0, int64_t pml_y0, int64_t pml_x0,         \
      int64_t pml_z1, int64_t pml_y1, int64_t pml_x1,                          \
      int64_t source_component, int64_t receiver_component, int64_t n_threads, \
      int64_t device, int64_t execution_backend, void *compute_stream

/* maxwell_3d_*_born_forward_with_storage_cuda.  Replaces
 * maxwell_3d_{S}_{dtype}_born_forward_with_storage_cuda,
 * src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:4045-4540 (argtypes
 * src/tide/backend_utils.py:579-612).  born_forward plus, at steps
 * t % step_ratio == 0 in device storage mode, the background E^n (when
 * ca_requires_grad) and CPML-corrected curl H^n (when cb_requires_grad) into
 * the s1 buffers, and the scattered E^n and curl into the dex_store ..
 * dcurl_z_store buffers that are not null; snapshot t sits at byte offset
 * (t / step_ratio) * n_shots * shot_bytes_uncomp.  Other storage modes store
 * nothing, as in the reference.  CPML memories are full arrays. */
#define TIDE_3D_BORN_FORWARD_WITH_STORAGE_ARGS(T)                              \
  T const *ca, T const *cb, T const *cq, T const *dca, T const *dcb,           \
      T const *f0, T const *df, T *ex, T *ey, T *ez, T *hx, T *hy, T *hz,      \
      T *m_hz_y, T *m_hy_z, T *m_hx_z, T *m_hz_x, T *m_hy_x, T *m_hx_y,        \
      T *m_ey_z, T *m_ez_y, T *m_ez_x, T *m_ex_z, T *m_ex_y, T *m_ey_x,        \
      T *dex, T *dey, T *dez, T *dhx, T *dhy, T *dhz, T *dm_hz_y, T *dm_hy_z,  \
      T *dm_hx_z, T *dm_hz_x, T *dm_hy_x, T *dm_hx_y, T *dm_ey_z, T *dm_ez_y,  \
      T *dm_ez_x, T *dm_ex_z, T *dm_ex_y, T *dm_ey_x, T *r, T *background_r,   \
      void *ex_s1, void *ex_s3, void *ex_fn, void *ey_s1, void *ey_s3,         \
      void *ey_fn, void *ez_s1, void *ez_s3, void *ez_fn, void *cx_s1,         \
      void *cx_s3, void *cx_fn, void *cy_s1, void *cy_s3, void *cy_fn,         \
      void *cz_s1, void *cz_s3, void *cz_fn, void *dex_store, void *dey_store, \
      void *dez_store, void *dcurl_x_store, void *dcurl_y_store,               \
      void *dcurl_z_store, T const *az, T const *bz, T const *azh,             \
      T const *bzh, T const *ay, T const *by, T const *ayh, T const *byh,      \
      T const *ax, T const *bx, T const *axh, T const *bxh, T const *kz,       \
      T const *kzh, T const *ky, T const *kyh, T const *kx, T const *kxh,      \
      int64_t const *sources_i, int64_t const *receivers_i, T rdz, T rdy,      \
      T rdx, T dt, int64_t nt, int64_t n_shots, int64_t nz, int64_t ny,        \
      int64_t nx, int64_t n_sources_per_shot, int64_t n_receivers_per_shot,    \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_z0, int64_t pml_y0, int64_t pml_x0, int64_t pml_z1,          \
      int64_t pml_y1, int64_t pml_x1, int64_t source_component,                \
      int64_t receiver_component, int64_t n_threads, int64_t device,           \
      int64_t execution_backend, void *compute_stream, void *storage_stream

/* maxwell_3d_*_born_backward_cuda.  Replaces
 * maxwell_3d_{S}_{dtype}_born_backward_cuda,
 * src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:5901-6290 (argtypes
 * src/tide/backend_utils.py:614-633).  The adjoint of the Born map with
 * respect to dca, dcb and the scattered sources: the exact adjoint of the
 * background operator driven by grad_r, imaging against the stored
 * background E^n / curl H^n into grad_ca / grad_cb (the gradients of dca /
 * dcb) and recording grad_f at the sources.  grad_f, grad_ca, grad_cb and
 * grad_*_shot are zeroed on entry; CPML memories and adjoint_memory_scratch
 * are full [S, nz, ny, nx] arrays (12 of them in the scratch). */
#define TIDE_3D_BORN_BACKWARD_ARGS(T)                                          \
  T const *ca, T const *cb, T const *cq, T const *grad_r, T *lambda_ex,        \
      T *lambda_ey, T *lambda_ez, T *lambda_hx, T *lambda_hy, T *lambda_hz,    \
      T *m_lambda_ey_z, T *m_lambda_ez_y, T *m_lambda_ez_x, T *m_lambda_ex_z,  \
      T *m_lambda_ex_y, T *m_lambda_ey_x, T *m_lambda_hz_y, T *m_lambda_hy_z,  \
      T *m_lambda_hx_z, T *m_lambda_hz_x, T *m_lambda_hy_x, T *m_lambda_hx_y,  \
      T *adjoint_memory_scratch, void *ex_s1, void *ex_s3, void *ex_fn,        \
      void *ey_s1, void *ey_s3, void *ey_fn, void *ez_s1, void *ez_s3,         \
      void *ez_fn, void *cx_s1, void *cx_s3, void *cx_fn, void *cy_s1,         \
      void *cy_s3, void *cy_fn, void *cz_s1, void *cz_s3, void *cz_fn,         \
      T *grad_f, T *grad_ca, T *grad_cb, T *grad_ca_shot, T *grad_cb_shot,     \
      T const *az, T const *bz, T const *azh, T const *bzh, T const *ay,       \
      T const *by, T const *ayh, T const *byh, T const *ax, T const *bx,       \
      T const *axh, T const *bxh, T const *kz, T const *kzh, T const *ky,      \
      T const *kyh, T const *kx, T const *kxh, int64_t const *sources_i,       \
      int64_t const *receivers_i, T rdz, T rdy, T rdx, T dt, int64_t nt,       \
      int64_t n_shots, int64_t nz, int64_t ny, int64_t nx,                     \
      int64_t n_sources_per_shot, int64_t n_receivers_per_shot,                \
      int64_t step_ratio, int64_t storage_mode, int64_t storage_format,        \
      int64_t shot_bytes_uncomp, bool ca_requires_grad, bool cb_requires_grad, \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_z0, int64_t pml_y0, int64_t pml_x0, int64_t pml_z1,          \
      int64_t pml_y1, int64_t pml_x1, int64_t source_component,                \
      int64_t receiver_component, int64_t n_threads, int64_t device,           \
      int64_t execution_backend, void *compute_stream, void *storage_stream

/* maxwell_3d_*_born_backward_bggrad_cuda.  Replaces
 * maxwell_3d_{S}_{dtype}_born_backward_bggrad_cuda,
 * src/tide/csrc/em3d/maxwell_3d_cuda_inst.cu:5262-5900 (argtypes
 * src/tide/backend_utils.py:635-671): the derivative of grad_r . (scattered
 * receivers) in the background coefficients (grad_ca, grad_cb), the
 * perturbation (grad_dca, grad_dcb) and both sources (grad_f0, grad_df), by
 * the exact adjoint of the joint background + scattered recurrence over the
 * background (s1) and scattered (dex_store ..) histories of
 * born_forward_with_storage, device storage mode.  lambda_* receive the
 * scattered state's adjoint, eta_* the background's (fields and full-size
 * memories, zeroed on entry); adjoint_memory_scratch holds 24 and
 * eta_source_e* one n_shots nz ny nx array each; gradients accumulate, per
 * shot into grad_*_shot (zeroed here) when several unbatched shots share the
 * model, then summed in shot order. */
#define TIDE_3D_BORN_BACKWARD_BGGRAD_ARGS(T)                                   \
  T const *ca, T const *cb, T const *cq, T const *dca, T const *dcb,           \
      T const *f0, T const *df, T const *grad_r, T *lambda_ex, T *lambda_ey,   \
      T *lambda_ez, T *lambda_hx, T *lambda_hy, T *lambda_hz,                  \
      T *m_lambda_ey_z, T *m_lambda_ez_y, T *m_lambda_ez_x, T *m_lambda_ex_z,  \
      T *m_lambda_ex_y, T *m_lambda_ey_x, T *m_lambda_hz_y, T *m_lambda_hy_z,  \
      T *m_lambda_hx_z, T *m_lambda_hz_x, T *m_lambda_hy_x, T *m_lambda_hx_y,  \
      T *eta_ex, T *eta_ey, T *eta_ez, T *eta_hx, T *eta_hy, T *eta_hz,        \
      T *m_eta_ey_z, T *m_eta_ez_y, T *m_eta_ez_x, T *m_eta_ex_z,              \
      T *m_eta_ex_y, T *m_eta_ey_x, T *m_eta_hz_y, T *m_eta_hy_z,              \
      T *m_eta_hx_z, T *m_eta_hz_x, T *m_eta_hy_x, T *m_eta_hx_y,              \
      T *adjoint_memory_scratch, void *ex_s1, void *ex_s3, void *ex_fn,        \
      void *ey_s1, void *ey_s3, void *ey_fn, void *ez_s1, void *ez_s3,         \
      void *ez_fn, void *cx_s1, void *cx_s3, void *cx_fn, void *cy_s1,         \
      void *cy_s3, void *cy_fn, void *cz_s1, void *cz_s3, void *cz_fn,         \
      void *dex_store, void *dey_store, void *dez_store, void *dcurl_x_store,  \
      void *dcurl_y_store, void *dcurl_z_store, T *grad_f0, T *grad_df,        \
      T *grad_ca, T *grad_cb, T *grad_dca, T *grad_dcb, T *grad_ca_shot,       \
      T *grad_cb_shot, T *grad_dca_shot, T *grad_dcb_shot, T *eta_source_ex,   \
      T *eta_source_ey, T *eta_source_ez, T const *az, T const *bz,            \
      T const *azh, T const *bzh, T const *ay, T const *by, T const *ayh,      \
      T const *byh, T const *ax, T const *bx, T const *axh, T const *bxh,      \
      T const *kz, T const *kzh, T const *ky, T const *kyh, T const *kx,       \
      T const *kxh, int64_t const *sources_i, int64_t const *receivers_i,      \
      T rdz, T rdy, T rdx, T dt, int64_t nt, int64_t n_shots, int64_t nz,      \
      int64_t ny, int64_t nx, int64_t n_sources_per_shot,                      \
      int64_t n_receivers_per_shot, int64_t step_ratio, int64_t storage_mode,  \
      int64_t storage_format, int64_t shot_bytes_uncomp, bool ca_requires_grad, \
      bool cb_requires_grad, bool dca_requires_grad, bool dcb_requires_grad,   \
      bool ca_batched, bool cb_batched, bool cq_batched, int64_t start_t,      \
      int64_t pml_z0, int64_t pml_y0, int64_t pml_x0, int64_t pml_z1,          \
      int64_t pml_y1, int64_t pml_x1, int64_t source_component,                \
      int64_t receiver_component, int64_t n_threads, int64_t device,           \
      int64_t execution_backend, void *compute_stream, void *storage_stream

#define TIDE_3D_BORN_DECLARE(S, T)                                              \
  void maxwell_3d_##S##_##T##_born_forward_cuda(TIDE_3D_BORN_FORWARD_ARGS(T)); \
  void maxwell_3d_##S##_##T##_born_forward_with_storage_cuda(                   \
      TIDE_3D_BORN_FORWARD_WITH_STORAGE_ARGS(T));                               \
  void maxwell_3d_##S##_##T##_born_backward_cuda(TIDE_3D_BORN_BACKWARD_ARGS(T));  \
  void maxwell_3d_##S##_##T##_born_backward_bggrad_cuda(                        \
      TIDE_3D_BORN_BACKWARD_BGGRAD_ARGS(T));
TIDE_3D_BORN_DECLARE(2, float)
TIDE_3D_BORN_DECLARE(2, double)
TIDE_3D_BORN_DECLARE(4, float)
TIDE_3D_BORN_DECLARE(4, double)
TIDE_3D_BORN_DECLARE(6, float)
TIDE_3D_BORN_DECLARE(6, double)
TIDE_3D_BORN_DECLARE(8, float)
TIDE_3D_BORN_DECLARE(8, double)

/* Comma-separated CUDA architectures the library was built for ("100a").
 * Replaces tide_cuda_arches, src/tide/csrc/storage/storage_utils.cu:213. */
const char *tide_cuda_arches(void);

/* Status of the most recent failed call in this process (0 = none) and its
 * message.  New: the reference exits the process instead
 * (src/tide/csrc/common/common_gpu.h:12-31). */
int tide_b200_last_status(void);
const char *tide_b200_last_error(void);
void tide_b200_clear_error(void);

/* Synchronises `device` and returns the device-side error word that kernels
 * set instead of faulting (e.g. a source index outside its shot), then clears
 * it.  0 = clean.  New; the reference has no device-side checks. */
int tide_b200_device_status(int64_t device);

/* Kernel timing for benchmarks (new; no reference counterpart).  When
 * enabled, every `sample_every`-th time step of each call brackets its stencil
 * kernels with CUDA events on the launching stream; durations accumulate per
 * kernel kind until read (reading waits for the recorded events; profiled
 * calls themselves never block).  Kinds: 0 fwd_h, 1 fwd_e, 2 adj_e, 3 adj_h,
 * 4 fwd_step (one-sweep forward), 5 adj_step (one-sweep adjoint), 6 em3d_fwd_h,
 * 7 em3d_fwd_e, 8 em3d_adj_e, 9 em3d_adj_h, 10 em3d_grad (3-D path). */
void tide_b200_profile_enable(int on, int sample_every);
int tide_b200_profile_read(double *ms_out, int64_t *launches_out, int max_kinds);
const char *tide_b200_profile_kind_name(int kind);

/* Total kernels this library has launched in this process (monotonic). */
int64_t tide_b200_launch_count(void);

/* Per-call scratch comes from the device's default stream-ordered memory
 * pool, which keeps up to 4 GiB of freed memory for later calls.  This waits
 * for the device and returns all of it to the driver (for a caller that
 * budgets device memory itself).  0 on success, -1 (status set) on error. */
int tide_b200_release_scratch(int64_t device);

/* Selection between the two stencil-2 FP32 forward implementations (new; no
 * reference counterpart).  A call whose three field arrays (3 * n_shots * ny
 * * nx * 4 bytes) exceed `bytes` runs the fused one-launch-per-step kernel;
 * smaller calls run the H/E kernel pair, whose re-reads then hit L2.  0 = always
 * fused, negative = never.  Default 64 MiB.  Returns the previous setting;
 * process-wide, takes effect at the next call. */
int64_t tide_b200_set_fused_threshold(int64_t bytes);

/* Selection of the one-sweep TMA time steps (new; no reference counterpart):
 * FP32 stencil-2 forward, forward_with_storage and backward with model
 * coefficients shared by the shots and no Debye poles run one launch per time
 * step on TMA-staged tiles (both half steps fused) on persistent CTAs.
 * 0 = never (default), 1 = when the grid has at least 64 tiles of 32 x 64
 * cells, 2 = whenever eligible.  Results are bit-identical in every mode.
 * Returns the previous mode; process-wide, takes effect at the next call. */
int tide_b200_set_tma_mode(int mode);

/* Upper bound on the persistent CTAs of the TMA time steps (new; no reference
 * counterpart): 0 = one per SM (default).  Smaller bounds give each CTA more
 * tiles and split more tiles between neighbouring CTAs; results are
 * bit-identical for every bound.  Returns the previous bound. */
int tide_b200_set_tma_ctas(int max_ctas);

/* Step blocks replayed from CUDA graphs (new; no reference counterpart): the
 * TM2D forward, forward_with_storage and backward of the per-cell kernels and
 * the Born forward, born_forward_with_storage, tangent and
 * born_backward_bggrad passes, with the
 * snapshot history on the device or none, run a call of at least
 * three blocks (64 steps, or the next multiple of the even snapshot
 * interval) as one captured graph replayed per block instead of two launches
 * per step; the step-indexed pointers move with a device-side block counter.
 * Results are bit-identical either way.  1 = on (default), 0 = off.  Returns
 * the previous setting; process-wide, takes effect at the next call. */
int tide_b200_set_step_graphs(int on);

/* Graph replays issued so far by this process (each one block of steps). */
int64_t tide_b200_graph_replays(void);

#ifdef __cplusplus
}
#endif

#endif /* TIDE_B200_H */
