/* Debye-medium TM2D gradient entry points of libtide_b200.so.
 *
 * The reference's native backends run Debye media forward only
 * (maxwell_tm_cuda_inst.cu:382-457, maxwell_tm_inst.cpp forward_kernel_e_debye)
 * and differentiate them in Python, by torch autograd through the whole time
 * loop (src/tide/maxwell/tm2d_python.py:440-503).  These two entry points have
 * no counterpart in the reference: a forward that records what the Debye
 * adjoint needs and the exact discrete adjoint of the Debye time step, with the
 * gradients of the update coefficients ca, cb and of the pole coefficients a,
 * b, cp accumulated in the adjoint sweep.
 *
 * Forward step (per cell of the update domain, poles p):
 *   e1 = ca E + cb curlH + sum_p cp_p P_p (+ sources)
 *   P_p <- a_p P_p + b_p (e1 + E);  E <- e1.
 * Adjoint state: g (adjoint of e1, held in lam[0]), lambda_H, the CPML
 * memory adjoints, lambda_P [S, n_poles, ny, nx].  Adjoint of step t:
 *   lambda_E  = ca g' + curl^T(...) + receivers' adjoint,  U = sum_p b_p lambda_P_p
 *   lambda_P_p <- a_p lambda_P_p + cp_p g'
 *   g = (lambda_E + U) + sum_p b_p lambda_P_p
 * and images  d ca += g E^t,  d cb += g curl^t,  d cp_p += g P_p^t,
 *             d a_p += lambda_P_p P_p^t,  d b_p += lambda_P_p (E^{t+1} + E^t),
 * each times the sampling interval k at stored steps (t % k == 0).
 *
 * Snapshot buffers hold store indices q0, q0+1, ... (q = t / k) of
 * [S, ny, nx] (Ey, curl H, E^{t+1} + E^t) or [S, n_poles, ny, nx] (P) each,
 * in float/double or bf16 (storage_format 1, float only).  Only the update
 * domain of each snapshot is written.  Models are not batched.  Every call
 * returns after enqueueing on `stream`; failures set tide_b200_last_status.
 */
#ifndef TIDE_B200_DEBYE_H
#define TIDE_B200_DEBYE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct TideTMDebye {
  int64_t stencil;  /* 2, 4, 6 or 8 */
  int64_t n_shots, ny, nx, nt, start_t, n_src, n_rec, n_poles, step_ratio;
  int64_t storage_format, q0;
  int64_t pml_y0, pml_x0, pml_y1, pml_x1;
  double rdy, rdx;
  /* CPML profiles: ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh */
  const void *profiles[12];
  const void *ca, *cb, *cq;      /* [ny, nx] */
  const void *a, *b, *cp;        /* [n_poles, ny, nx] */
  void *fields[7];               /* Ey, Hx, Hz, m_Ey_x, m_Ey_z, m_Hx_z, m_Hz_x [S, ny, nx] */
  void *pol;                     /* [S, n_poles, ny, nx] */
  const void *f;                 /* [nt, S, n_src] scaled source amplitudes */
  void *r;                       /* [nt, S, n_rec] */
  const int64_t *sources_i, *receivers_i;
  void *ey_store, *curl_store, *pol_store, *esum_store; /* any may be null */
  /* adjoint */
  const void *grad_r;            /* [nt, S, n_rec] */
  void *lam[7];                  /* g, lambda_Hx, lambda_Hz, memory adjoints (as fields) */
  void *lam_pol;                 /* [S, n_poles, ny, nx] */
  void *scratch;                 /* [5, S, ny, nx] */
  void *grad_f;                  /* [nt, S, n_src] or null */
  void *grad_ca, *grad_cb;       /* [ny, nx], accumulated into; null to skip */
  void *grad_cp, *grad_a, *grad_b; /* [n_poles, ny, nx], accumulated into; null to skip */
  int64_t device;
  void *stream;
} TideTMDebye;

/* Forward over steps start_t .. start_t + nt - 1, recording the snapshots whose
 * buffers are given; fields and pol advance in place. */
void tide_b200_tm_debye_forward_with_storage_float(const TideTMDebye *args);
void tide_b200_tm_debye_forward_with_storage_double(const TideTMDebye *args);
/* Adjoint over steps start_t - 1 down to start_t - nt (chained calls continue
 * the adjoint state held in lam, lam_pol).  The snapshots of those steps must
 * be in the store buffers. */
void tide_b200_tm_debye_backward_float(const TideTMDebye *args);
void tide_b200_tm_debye_backward_double(const TideTMDebye *args);

#ifdef __cplusplus
}
#endif

#endif /* TIDE_B200_DEBYE_H */
