// Debye-medium TM2D forward with storage and exact adjoint (interface and
// recursion: include/tide_b200_debye.h).  Included by tm2d_abi.cu: the sweeps
// reuse its per-call launch helpers, so the E/H parts of a Debye step are the
// same kernels as for a plain medium.
//
// Per adjoint step, after the adjoint E-phase (which reads g from lam[0]):
//   k_debye_pre    lambda_P <- a lambda_P + cp g,  U = sum_p b_p lambda_P(old)
//   adjoint H      lam[0] <- ca g + curl^T(...) + receivers' adjoint
//   k_debye_post   g <- (lam[0] + U) + sum_p b_p lambda_P;  all images
//   k_debye_gradf  source gradient = g at the source cells
// The pole kernels touch the update domain only, where the forward applies the
// pole terms.  Images are summed over shots in shot order, then added to the
// model-shaped gradients (one read-modify-write per cell and stored step).
#pragma once

#include "../../include/tide_b200_debye.h"

namespace tb {
namespace {

template <int ST>
__device__ __forceinline__ bool debye_dom(int64_t j, int ny, int nx) {
  constexpr int P = FD<ST>::P;
  const int y = (int)(j / nx), x = (int)(j % nx);
  return y >= P && y < ny - P + 1 && x >= P && x < nx - P + 1;
}

template <typename T, int ST>
__global__ void __launch_bounds__(256)
k_debye_pre(int ny, int nx, int n_poles, const T *__restrict__ a, const T *__restrict__ b,
            const T *__restrict__ cp, const T *__restrict__ g, T *__restrict__ lpol,
            T *__restrict__ U) {
  const int64_t N = (int64_t)ny * nx;
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (j >= N || !debye_dom<ST>(j, ny, nx)) return;
  const int64_t i = (int64_t)s * N + j;
  const T gv = g[i];
  T u = (T)0;
  for (int p = 0; p < n_poles; ++p) {
    const int64_t c = (int64_t)p * N + j, pi = ((int64_t)s * n_poles + p) * N + j;
    const T lp = lpol[pi];
    u = u + ldg(b + c) * lp;
    lpol[pi] = ldg(a + c) * lp + ldg(cp + c) * gv;
  }
  U[i] = u;
}

template <typename T> struct DebyeImages {
  const void *ey_st, *cu_st, *pol_st, *esum_st;  // this step's snapshots (null: none)
  T *grad_ca, *grad_cb, *grad_cp, *grad_a, *grad_b;
  T kscale;
};

template <typename T, int ST, typename S>
__global__ void __launch_bounds__(256)
k_debye_post(int ny, int nx, int n_shots, int n_poles, const T *__restrict__ b,
             const T *__restrict__ lpol, const T *__restrict__ U, T *__restrict__ g,
             DebyeImages<T> im) {
  const int64_t N = (int64_t)ny * nx;
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= N || !debye_dom<ST>(j, ny, nx)) return;
  const S *es = static_cast<const S *>(im.ey_st), *cs = static_cast<const S *>(im.cu_st);
  T sca = (T)0, scb = (T)0;
  for (int s = 0; s < n_shots; ++s) {
    const int64_t i = (int64_t)s * N + j;
    T sb = (T)0;
    for (int p = 0; p < n_poles; ++p)
      sb = sb + ldg(b + (int64_t)p * N + j) * lpol[((int64_t)s * n_poles + p) * N + j];
    const T gv = (g[i] + U[i]) + sb;
    g[i] = gv;
    if (es && im.grad_ca) sca = sca + gv * Codec<S, T>::dec(load_stream(es + i)) * im.kscale;
    if (cs && im.grad_cb) scb = scb + gv * Codec<S, T>::dec(load_stream(cs + i)) * im.kscale;
  }
  if (es && im.grad_ca) im.grad_ca[j] = im.grad_ca[j] + sca;
  if (cs && im.grad_cb) im.grad_cb[j] = im.grad_cb[j] + scb;
  const S *ps = static_cast<const S *>(im.pol_st), *qs = static_cast<const S *>(im.esum_st);
  for (int p = 0; p < n_poles; ++p) {
    if (ps && (im.grad_cp || im.grad_a)) {
      T scp = (T)0, sa = (T)0;
      for (int s = 0; s < n_shots; ++s) {
        const int64_t pi = ((int64_t)s * n_poles + p) * N + j;
        const T pv = Codec<S, T>::dec(load_stream(ps + pi));
        scp = scp + g[(int64_t)s * N + j] * pv * im.kscale;
        sa = sa + lpol[pi] * pv * im.kscale;
      }
      if (im.grad_cp) im.grad_cp[(int64_t)p * N + j] = im.grad_cp[(int64_t)p * N + j] + scp;
      if (im.grad_a) im.grad_a[(int64_t)p * N + j] = im.grad_a[(int64_t)p * N + j] + sa;
    }
    if (qs && im.grad_b) {
      T sbv = (T)0;
      for (int s = 0; s < n_shots; ++s)
        sbv = sbv + lpol[((int64_t)s * n_poles + p) * N + j] *
                        Codec<S, T>::dec(load_stream(qs + (int64_t)s * N + j)) * im.kscale;
      im.grad_b[(int64_t)p * N + j] = im.grad_b[(int64_t)p * N + j] + sbv;
    }
  }
}

template <typename T>
__global__ void k_debye_gradf(const int64_t *__restrict__ idx, int n_per_shot, int n_shots,
                              int64_t N, const T *__restrict__ g, T *__restrict__ gf_t) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_per_shot * n_shots) return;
  const int64_t v = idx[e];
  if (v < 0 || v >= N) return;
  gf_t[e] = g[(int64_t)(e / n_per_shot) * N + v];
}

template <typename T, int ST>
bool debye_setup(Launch<T, ST> &L, const TideTMDebye &A) {
  const T *const *pr = reinterpret_cast<const T *const *>(A.profiles);
  return make_launch(L, pr[0], pr[1], pr[2], pr[3], pr[4], pr[5], pr[6], pr[7], pr[8], pr[9],
                     pr[10], pr[11], (T)A.rdy, (T)A.rdx, A.n_shots, A.ny, A.nx, A.pml_y0,
                     A.pml_x0, A.pml_y1, A.pml_x1, false, false, false);
}

template <typename T>
bool debye_check(const TideTMDebye &A, bool adjoint) {
  if (A.n_poles < 1 || A.n_poles > 64 || A.step_ratio < 1 || A.nt < 0 || A.start_t < 0 ||
      (adjoint && A.start_t - A.nt < 0) || A.q0 < 0) {
    set_error(kBadArgument, "TM2D Debye: bad n_poles/step_ratio/nt/start_t/q0");
    return false;
  }
  if (A.storage_format != 0 && !(A.storage_format == 1 && sizeof(T) == 4)) {
    set_error(kBadArgument, "TM2D Debye: storage_format must be 0, or 1 (bf16) for float");
    return false;
  }
  if (!A.ca || !A.cb || !A.cq || !A.a || !A.b || !A.cp) {
    set_error(kBadArgument, "TM2D Debye: a coefficient pointer is null");
    return false;
  }
  for (int k = 0; k < 7; ++k)
    if (!(adjoint ? A.lam[k] : A.fields[k])) {
      set_error(kBadArgument, "TM2D Debye: state array %d is null", k);
      return false;
    }
  if (adjoint ? (!A.lam_pol || !A.scratch || (A.n_rec > 0 && !A.grad_r)) : !A.pol) {
    set_error(kBadArgument, "TM2D Debye: polarisation or adjoint buffers missing");
    return false;
  }
  if ((A.n_src > 0 && !A.sources_i) || (A.n_rec > 0 && !A.receivers_i) ||
      (!adjoint && ((A.n_src > 0 && !A.f) || (A.n_rec > 0 && !A.r)))) {
    set_error(kBadArgument, "TM2D Debye: sources/receivers without their buffers");
    return false;
  }
  return true;
}

template <typename T, int ST, typename S>
void debye_forward(const TideTMDebye &A) {
  if (TB_CUDA(cudaSetDevice((int)A.device))) return;
  if (!debye_check<T>(A, false)) return;
  Launch<T, ST> L;
  if (!debye_setup(L, A)) return;
  if (!L.has_domain) {
    set_error(kBadArgument, "TM2D Debye: grid has no update domain");
    return;
  }
  cudaStream_t st = as_stream(A.stream);
  PointScratch ps;
  if (!build_points(ps, L, PointTiles{L.tiles_x, L.tiles_y_e, kTileX, kBlockY * kRowsE, 0},
                    A.sources_i, A.n_src, A.receivers_i, A.n_rec, st))
    return;
  T *const *fld = reinterpret_cast<T *const *>(A.fields);
  const T *ca = static_cast<const T *>(A.ca), *cb = static_cast<const T *>(A.cb);
  const T *cq = static_cast<const T *>(A.cq);
  const int64_t SN = A.n_shots * A.ny * A.nx, np = A.n_poles;
  const int64_t fs = A.n_shots * A.n_src, rs = A.n_shots * A.n_rec;
  const T *f = static_cast<const T *>(A.f);
  T *r = static_cast<T *>(A.r);
  for (int64_t t = A.start_t; t < A.start_t + A.nt; ++t) {
    const bool store = t % A.step_ratio == 0;
    const int64_t q = t / A.step_ratio - A.q0;
    auto at = [&](void *base, int64_t per) -> void * {
      return store && base ? static_cast<void *>(static_cast<S *>(base) + q * per) : nullptr;
    };
    DebyeArgs<T> db{static_cast<const T *>(A.a), static_cast<const T *>(A.b),
                    static_cast<const T *>(A.cp), static_cast<T *>(A.pol), (int)np,
                    at(A.pol_store, SN * np), at(A.esum_store, SN)};
    launch_fwd_h<T, ST>(L, st, cq, fld[0], fld[1], fld[2], fld[3], fld[4]);
    k_fwd_e<T, ST, S, kRowsE><<<L.grid_e, L.block, 0, st>>>(
        L.g, ca, cb, fld[1], fld[2], fld[0], fld[5], fld[6], static_cast<S *>(at(A.ey_store, SN)),
        static_cast<S *>(at(A.curl_store, SN)), db, ps.src, ps.rec, f ? f + t * fs : nullptr,
        r ? r + t * rs : nullptr, StepShift{});
  }
  count_launches(2 * A.nt);
  TB_CUDA(cudaGetLastError());
}

template <typename T, int ST, typename S>
void debye_backward(const TideTMDebye &A) {
  if (TB_CUDA(cudaSetDevice((int)A.device))) return;
  if (!debye_check<T>(A, true)) return;
  Launch<T, ST> L;
  if (!debye_setup(L, A)) return;
  if (!L.has_domain) {
    set_error(kBadArgument, "TM2D Debye: grid has no update domain");
    return;
  }
  cudaStream_t st = as_stream(A.stream);
  const int64_t N = A.ny * A.nx, SN = A.n_shots * N, np = A.n_poles;
  T *const *lam = reinterpret_cast<T *const *>(A.lam);
  T *scratch = static_cast<T *>(A.scratch);
  if (TB_CUDA(cudaMemsetAsync(scratch, 0, 5 * SN * sizeof(T), st))) return;
  if (!zero_band(lam[6], L.g, 1, L.g.pml_x0, L.g.pml_x1, st) ||
      !zero_band(lam[5], L.g, 0, L.g.pml_y0, L.g.pml_y1, st) ||
      !zero_band(lam[3], L.g, 1, L.g.pml_x0, L.g.pml_x1h, st) ||
      !zero_band(lam[4], L.g, 0, L.g.pml_y0, L.g.pml_y1h, st))
    return;
  PointScratch ps;
  if constexpr (ST == 2) pick_adj_h_rows<T, T>(L);
  L.narrow_e();  // 4-warp adjoint E blocks (the adjoint E kernel has no point lists)
  if (!build_points(ps, L, L.ah_tiles(), A.sources_i, A.n_src, A.receivers_i, A.n_rec, st))
    return;
  const T *ca = static_cast<const T *>(A.ca), *cb = static_cast<const T *>(A.cb);
  const T *cq = static_cast<const T *>(A.cq);
  const T *da = static_cast<const T *>(A.a), *db = static_cast<const T *>(A.b);
  const T *dcp = static_cast<const T *>(A.cp);
  T *lpol = static_cast<T *>(A.lam_pol);
  T *U = scratch + 4 * SN;
  T *cur_ey_x = lam[3], *cur_ey_z = lam[4], *cur_hx_z = lam[5], *cur_hz_x = lam[6];
  T *nxt_ey_x = scratch, *nxt_ey_z = scratch + SN;
  T *nxt_hx_z = scratch + 2 * SN, *nxt_hz_x = scratch + 3 * SN;
  const int64_t fs = A.n_shots * A.n_src, rs = A.n_shots * A.n_rec;
  const T *grad_r = static_cast<const T *>(A.grad_r);
  T *grad_f = static_cast<T *>(A.grad_f);
  const dim3 pgrid((unsigned)((N + 255) / 256), (unsigned)A.n_shots);
  const unsigned cgrid = (unsigned)((N + 255) / 256);
  const GradArgs<T, T> none{nullptr, nullptr, nullptr, nullptr, (T)1, false, false};
  for (int64_t t = A.start_t - 1; t >= A.start_t - A.nt; --t) {
    launch_adj_e<T, ST>(L, st, cb, lam[0], lam[1], lam[2], cur_hx_z, cur_hz_x, nxt_hx_z,
                        nxt_hz_x);
    std::swap(cur_hx_z, nxt_hx_z);
    std::swap(cur_hz_x, nxt_hz_x);
    k_debye_pre<T, ST><<<pgrid, 256, 0, st>>>((int)A.ny, (int)A.nx, (int)np, da, db, dcp, lam[0],
                                              lpol, U);
    launch_adj_h<T, ST, T>(L, st, ca, cq, lam[1], lam[2], lam[0], cur_ey_x, cur_ey_z, nxt_ey_x,
                           nxt_ey_z, ps, grad_r ? grad_r + t * rs : nullptr, nullptr, none);
    std::swap(cur_ey_x, nxt_ey_x);
    std::swap(cur_ey_z, nxt_ey_z);
    const bool img = t % A.step_ratio == 0;
    const int64_t q = t / A.step_ratio - A.q0;
    auto at = [&](void *base, int64_t per) -> const void * {
      return img && base ? static_cast<const void *>(static_cast<S *>(base) + q * per) : nullptr;
    };
    DebyeImages<T> im{at(A.ey_store, SN), at(A.curl_store, SN), at(A.pol_store, SN * np),
                      at(A.esum_store, SN), static_cast<T *>(A.grad_ca),
                      static_cast<T *>(A.grad_cb), static_cast<T *>(A.grad_cp),
                      static_cast<T *>(A.grad_a), static_cast<T *>(A.grad_b),
                      (T)A.step_ratio};
    k_debye_post<T, ST, S><<<cgrid, 256, 0, st>>>((int)A.ny, (int)A.nx, (int)A.n_shots, (int)np,
                                                  db, lpol, U, lam[0], im);
    if (A.n_src > 0 && grad_f) {
      const int n = (int)(A.n_src * A.n_shots);
      k_debye_gradf<T><<<(n + 255) / 256, 256, 0, st>>>(A.sources_i, (int)A.n_src,
                                                        (int)A.n_shots, N, lam[0],
                                                        grad_f + t * fs);
    }
  }
  const size_t nb = SN * sizeof(T);
  if (cur_ey_x != lam[3]) {
    if (TB_CUDA(cudaMemcpyAsync(lam[3], cur_ey_x, nb, cudaMemcpyDeviceToDevice, st)) ||
        TB_CUDA(cudaMemcpyAsync(lam[4], cur_ey_z, nb, cudaMemcpyDeviceToDevice, st)) ||
        TB_CUDA(cudaMemcpyAsync(lam[5], cur_hx_z, nb, cudaMemcpyDeviceToDevice, st)) ||
        TB_CUDA(cudaMemcpyAsync(lam[6], cur_hz_x, nb, cudaMemcpyDeviceToDevice, st)))
      return;
  }
  count_launches(A.nt * (A.n_src > 0 && grad_f ? 5 : 4));
  TB_CUDA(cudaGetLastError());
}

template <typename T, bool kFwd>
void debye_dispatch(const TideTMDebye *A) {
  if (A == nullptr) {
    set_error(kBadArgument, "TM2D Debye: null argument struct");
    return;
  }
  const bool bf = A->storage_format == 1 && sizeof(T) == 4;
  using B = __nv_bfloat16;
#define TB_DEBYE_CASE(ST)                                                        \
  case ST:                                                                       \
    if (kFwd) {                                                                  \
      if (bf) debye_forward<T, ST, B>(*A);                                       \
      else debye_forward<T, ST, T>(*A);                                          \
    } else {                                                                     \
      if (bf) debye_backward<T, ST, B>(*A);                                      \
      else debye_backward<T, ST, T>(*A);                                         \
    }                                                                            \
    return;
  switch (A->stencil) {
    TB_DEBYE_CASE(2)
    TB_DEBYE_CASE(4)
    TB_DEBYE_CASE(6)
    TB_DEBYE_CASE(8)
    default:
      set_error(kBadArgument, "TM2D Debye: unsupported stencil %lld", (long long)A->stencil);
  }
#undef TB_DEBYE_CASE
}

}  // namespace
}  // namespace tb

extern "C" {
void tide_b200_tm_debye_forward_with_storage_float(const TideTMDebye *a) {
  tb::debye_dispatch<float, true>(a);
}
void tide_b200_tm_debye_forward_with_storage_double(const TideTMDebye *a) {
  tb::debye_dispatch<double, true>(a);
}
void tide_b200_tm_debye_backward_float(const TideTMDebye *a) {
  tb::debye_dispatch<float, false>(a);
}
void tide_b200_tm_debye_backward_double(const TideTMDebye *a) {
  tb::debye_dispatch<double, false>(a);
}
}
