// Born (tangent) propagation of the TM2D path: the background state and the
// scattered state advance together (maxwell_tm_cuda_inst.cu:1611-1703,
// maxwell_tm_core.cuh:601-690).  Included by tm2d_abi.cu: both H half-steps
// are the forward H kernel on the two states; one E kernel updates both
// states, the scattered one with the extra terms dca Ey^n + dcb curl H^n of
// the background, then injects the background sources (f0) and the
// scattered sources (df) and records both states at the receivers.  Every
// expression keeps the reference's operation order, so with the same inputs
// the results are bit-identical to its CPU backend.
//
// The storing Born forward (cu_inst:1701-2086) runs the same steps through the
// snapshot pipeline of forward_with_storage (StoreRun), storing the
// background Ey^n / curl H^n and, when asked, the scattered dEy^n / dcurl H^n.
// The Born backward for (dca, dcb, df) (cu_inst:2088-2400) is the ordinary
// adjoint over the background history: the scattered update is linear in
// (dca, dcb, df) with factors Ey^n, curl H^n and the source weights, which
// are the factors of (ca, cb, f) in the background update.
#pragma once

namespace tb {
namespace {

// Born E half-step.  Full-grid tiles of 32 x 8R (as k_fwd_e) so point
// entries outside the update domain are still served.  Non-null store
// pointers (this step's slots, type S) receive Ey^n, curl H^n, dEy^n and
// dcurl H^n of the update domain.
template <typename T, int ST, typename S, int R, int BY = kBlockY>
__global__ void __launch_bounds__(32 * BY)
k_born_e(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cb,
         const T *__restrict__ dca, const T *__restrict__ dcb, const T *__restrict__ hx,
         const T *__restrict__ hz, T *__restrict__ ey, T *__restrict__ m_hx_z,
         T *__restrict__ m_hz_x, const T *__restrict__ dhx, const T *__restrict__ dhz,
         T *__restrict__ dey, T *__restrict__ dm_hx_z, T *__restrict__ dm_hz_x, PointCSR src,
         PointCSR rec, const T *__restrict__ f0_t, const T *__restrict__ df_t,
         T *__restrict__ r_t, T *__restrict__ bgr_t, S *__restrict__ es,
         S *__restrict__ cs, S *__restrict__ des, S *__restrict__ dcs, StepShift sh) {
  constexpr int P = FD<ST>::P;
  if (sh.blk) {
    const int64_t jb = sh.block();
    f0_t = shifted(f0_t, sh.src, jb);
    df_t = shifted(df_t, sh.src, jb);
    r_t = shifted(r_t, sh.rec, jb);
    bgr_t = shifted(bgr_t, sh.rec, jb);
    es = shifted(es, sh.snap, jb);
    cs = shifted(cs, sh.snap, jb);
    des = shifted(des, sh.snap, jb);
    dcs = shifted(dcs, sh.snap, jb);
  }
  const int x = blockIdx.x * kTileX + threadIdx.x;
  const int y0 = (blockIdx.y * BY + threadIdx.y) * R;
  const int s = blockIdx.z;
  const int tile = (s * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const bool pts = !point_tile_empty(src, rec, tile);
  if (x >= g.nx || y0 >= g.ny) return;
  const int64_t base = (int64_t)s * g.N;
  const bool xdom = x >= P && x < g.nx - P + 1;
  const bool px = x < g.pml_x0 || x >= g.pml_x1;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    if (y >= g.ny) break;
    const bool dom = xdom && y >= P && y < g.ny - P + 1;
    if (!dom && !pts) continue;
    const int64_t j = (int64_t)y * g.nx + x, i = base + j;
    T e = ey[i], de = dey[i];
    if (dom) {
      const T cav = g.ca_b ? ldg(ca + i) : ldg(ca + j);
      const T cbv = g.cb_b ? ldg(cb + i) : ldg(cb + j);
      const T dcav = g.ca_b ? ldg(dca + i) : ldg(dca + j);
      const T dcbv = g.cb_b ? ldg(dcb + i) : ldg(dcb + j);
      T dz = d_x1<T, ST>(hz, i, g.rdx), dy = d_y1<T, ST>(hx, i, g.nx, g.rdy);
      T ddz = d_x1<T, ST>(dhz, i, g.rdx), ddy = d_y1<T, ST>(dhx, i, g.nx, g.rdy);
      if (px) {
        const T bxv = ldg(g.bx + x), axv = ldg(g.ax + x), kxv = ldg(g.kx + x);
        const T m = bxv * m_hz_x[i] + axv * dz;
        m_hz_x[i] = m;
        dz = dz / kxv + m;
        const T dm = bxv * dm_hz_x[i] + axv * ddz;
        dm_hz_x[i] = dm;
        ddz = ddz / kxv + dm;
      }
      if (y < g.pml_y0 || y >= g.pml_y1) {
        const T byv = ldg(g.by + y), ayv = ldg(g.ay + y), kyv = ldg(g.ky + y);
        const T m = byv * m_hx_z[i] + ayv * dy;
        m_hx_z[i] = m;
        dy = dy / kyv + m;
        const T dm = byv * dm_hx_z[i] + ayv * ddy;
        dm_hx_z[i] = dm;
        ddy = ddy / kyv + dm;
      }
      const T curl = dz - dy, dcurl = ddz - ddy;
      const T e_n = e, de_n = de;
      if (es) store_stream(es + i, Codec<S, T>::enc(e_n));
      if (cs) store_stream(cs + i, Codec<S, T>::enc(curl));
      if (des) store_stream(des + i, Codec<S, T>::enc(de_n));
      if (dcs) store_stream(dcs + i, Codec<S, T>::enc(dcurl));
      e = cav * e_n + cbv * curl;
      de = cav * de_n + cbv * dcurl + dcav * e_n + dcbv * curl;
    }
    if (pts) {
      e = point_accumulate(src, tile, (int)j, f0_t, e);
      de = point_accumulate(src, tile, (int)j, df_t, de);
    }
    ey[i] = e;
    dey[i] = de;
    if (pts) {
      point_record(rec, tile, (int)j, r_t, de);
      point_record(rec, tile, (int)j, bgr_t, e);
    }
  }
}

// Scattered E half-step from a stored background history
// (maxwell_tm_core.cuh:691-743): Ey^n and curl H^n of background shot
// s % bg_shots are read from this step's slots e_bg / c_bg (type S) instead
// of being recomputed; then the scattered sources and receivers.
template <typename T, int ST, typename S, int R, int BY = kBlockY>
__global__ void __launch_bounds__(32 * BY)
k_born_tangent_e(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cb,
                 const T *__restrict__ dca, const T *__restrict__ dcb,
                 const T *__restrict__ dhx, const T *__restrict__ dhz, T *__restrict__ dey,
                 T *__restrict__ dm_hx_z, T *__restrict__ dm_hz_x, const S *__restrict__ e_bg,
                 const S *__restrict__ c_bg, int bg_shots, PointCSR src, PointCSR rec,
                 const T *__restrict__ df_t, T *__restrict__ r_t, S *__restrict__ des,
                 S *__restrict__ dcs, StepShift sh) {
  constexpr int P = FD<ST>::P;
  if (sh.blk) {
    const int64_t jb = sh.block();
    df_t = shifted(df_t, sh.src, jb);
    r_t = shifted(r_t, sh.rec, jb);
    e_bg = shifted(e_bg, sh.hist, jb);
    c_bg = shifted(c_bg, sh.hist, jb);
    des = shifted(des, sh.snap, jb);
    dcs = shifted(dcs, sh.snap, jb);
  }
  const int x = blockIdx.x * kTileX + threadIdx.x;
  const int y0 = (blockIdx.y * BY + threadIdx.y) * R;
  const int s = blockIdx.z;
  const int tile = (s * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  const bool pts = !point_tile_empty(src, rec, tile);
  if (x >= g.nx || y0 >= g.ny) return;
  const int64_t base = (int64_t)s * g.N, bg_base = (int64_t)(s % bg_shots) * g.N;
  const bool xdom = x >= P && x < g.nx - P + 1;
  const bool px = x < g.pml_x0 || x >= g.pml_x1;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int y = y0 + r;
    if (y >= g.ny) break;
    const bool dom = xdom && y >= P && y < g.ny - P + 1;
    if (!dom && !pts) continue;
    const int64_t j = (int64_t)y * g.nx + x, i = base + j;
    T de = dey[i];
    if (dom) {
      const T cav = g.ca_b ? ldg(ca + i) : ldg(ca + j);
      const T cbv = g.cb_b ? ldg(cb + i) : ldg(cb + j);
      const T dcav = g.ca_b ? ldg(dca + i) : ldg(dca + j);
      const T dcbv = g.cb_b ? ldg(dcb + i) : ldg(dcb + j);
      T ddz = d_x1<T, ST>(dhz, i, g.rdx), ddy = d_y1<T, ST>(dhx, i, g.nx, g.rdy);
      if (px) {
        const T dm = ldg(g.bx + x) * dm_hz_x[i] + ldg(g.ax + x) * ddz;
        dm_hz_x[i] = dm;
        ddz = ddz / ldg(g.kx + x) + dm;
      }
      if (y < g.pml_y0 || y >= g.pml_y1) {
        const T dm = ldg(g.by + y) * dm_hx_z[i] + ldg(g.ay + y) * ddy;
        dm_hx_z[i] = dm;
        ddy = ddy / ldg(g.ky + y) + dm;
      }
      const T dcurl = ddz - ddy;
      const T de_n = de;
      const T e_n = Codec<S, T>::dec(e_bg[bg_base + j]);
      const T curl = Codec<S, T>::dec(c_bg[bg_base + j]);
      if (des) store_stream(des + i, Codec<S, T>::enc(de_n));
      if (dcs) store_stream(dcs + i, Codec<S, T>::enc(dcurl));
      de = cav * de_n + cbv * dcurl + dcav * e_n + dcbv * curl;
    }
    if (pts) de = point_accumulate(src, tile, (int)j, df_t, de);
    dey[i] = de;
    if (pts) point_record(rec, tile, (int)j, r_t, de);
  }
}

// Born E launches with the block shape of L (Launch::narrow_e: 4-warp blocks
// for stencil 2, whose point lists then follow L.e_tiles()).
template <typename T, int ST, typename S, typename... A>
inline void launch_born_e(const Launch<T, ST> &L, cudaStream_t s, A... a) {
  constexpr int NB = Launch<T, ST>::kNarrowBY;
  if (L.e_by == NB)
    k_born_e<T, ST, S, kRowsE, NB><<<L.grid_e_n, dim3(kTileX, NB, 1), 0, s>>>(a...);
  else
    k_born_e<T, ST, S, kRowsE><<<L.grid_e, L.block, 0, s>>>(a...);
}
template <typename T, int ST, typename S, typename... A>
inline void launch_born_tangent_e(const Launch<T, ST> &L, cudaStream_t s, A... a) {
  constexpr int NB = Launch<T, ST>::kNarrowBY;
  if (L.e_by == NB)
    k_born_tangent_e<T, ST, S, kRowsE, NB><<<L.grid_e_n, dim3(kTileX, NB, 1), 0, s>>>(a...);
  else
    k_born_tangent_e<T, ST, S, kRowsE><<<L.grid_e, L.block, 0, s>>>(a...);
}

template <typename T, int ST>
void tm_born_forward(TIDE_TM_BORN_FORWARD_ARGS(T)) {
  (void)dt; (void)step_ratio; (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0, "TM2D born_forward: nt must be >= 0");
  TB_REQUIRE(ca && cb && cq && dca && dcb && ey && hx && hz && m_ey_x && m_ey_z && m_hx_z &&
                 m_hz_x && dey && dhx && dhz && dm_ey_x && dm_ey_z && dm_hx_z && dm_hz_x,
             "TM2D born_forward: a field, memory or coefficient pointer is null");
  TB_REQUIRE(n_sources_per_shot == 0 || (f0 && df),
             "TM2D born_forward: sources without background or scattered amplitudes");
  TB_REQUIRE(n_receivers_per_shot == 0 || r, "TM2D born_forward: receivers without output");
  Launch<T, ST> L;
  if (!make_launch(L, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, rdy, rdx, n_shots,
                   ny, nx, pml_y0, pml_x0, pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  cudaStream_t st = as_stream(compute_stream);
  PointScratch ps;
  L.narrow_e();
  if (!build_points(ps, L, L.e_tiles(),
                    sources_i, n_sources_per_shot, receivers_i, n_receivers_per_shot, st))
    return;
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  ProfileScope prof(st);
  auto step = [&](int64_t i, cudaStream_t s, const int64_t *blk, int64_t B, bool) -> bool {
    const int64_t t = start_t + i;
    if (L.has_domain) {
      launch_fwd_h<T, ST>(L, s, cq, ey, hx, hz, m_ey_x, m_ey_z);
      launch_fwd_h<T, ST>(L, s, cq, dey, dhx, dhz, dm_ey_x, dm_ey_z);
    }
    launch_born_e<T, ST, T>(L, s,
        L.g, ca, cb, dca, dcb, hx, hz, ey, m_hx_z, m_hz_x, dhx, dhz, dey, dm_hx_z, dm_hz_x,
        ps.src, ps.rec, f0 ? f0 + t * fs : nullptr, df ? df + t * fs : nullptr,
        r ? r + t * rs : nullptr, background_r ? background_r + t * rs : nullptr, nullptr,
        nullptr, nullptr, nullptr, StepShift{blk, B * fs, B * rs, 0, 0});
    return true;
  };
  if (!run_step_blocks(nt, 1, st, prof, t_up, start_t, step)) return;
  count_launches(nt * (L.has_domain ? 3 : 1));
  TB_CUDA(cudaGetLastError());
}

template <typename T, int ST>
void tm_born_forward_with_storage(TIDE_TM_BORN_FORWARD_WITH_STORAGE_ARGS(T)) {
  (void)dt; (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1, "TM2D born_forward_with_storage: bad nt/step_ratio");
  TB_REQUIRE(ca && cb && cq && dca && dcb && ey && hx && hz && m_ey_x && m_ey_z && m_hx_z &&
                 m_hz_x && dey && dhx && dhz && dm_ey_x && dm_ey_z && dm_hx_z && dm_hz_x,
             "TM2D born_forward_with_storage: a field, memory or coefficient pointer is null");
  TB_REQUIRE(n_sources_per_shot == 0 || (f0 && df),
             "TM2D born_forward_with_storage: sources without background or scattered amplitudes");
  TB_REQUIRE(n_receivers_per_shot == 0 || r,
             "TM2D born_forward_with_storage: receivers without output");
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
  PointScratch ps;
  L.narrow_e();
  if (!build_points(ps, L, L.e_tiles(),
                    sources_i, n_sources_per_shot, receivers_i, n_receivers_per_shot, st))
    return;
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  const int64_t snap =
      sr.want ? (int64_t)(sr.step_bytes / (sr.bf16 ? sizeof(__nv_bfloat16) : sizeof(T))) : 0;
  ProfileScope prof(st);
  auto step = [&](int64_t i, cudaStream_t s, const int64_t *blk, int64_t B, bool) -> bool {
    const int64_t t = start_t + i;
    const StepShift sh{blk, B * fs, B * rs, B / step_ratio * snap, 0};
    char *dst[2];
    if (!sr.begin(t, dst)) return false;
    char *const e1 = dst[0], *const c1 = dst[1];
    // scattered history: device-resident, indexed by store index
    char *de1 = nullptr, *dc1 = nullptr;
    if (sr.stores(t)) {
      const size_t off = (size_t)(t / step_ratio) * sr.step_bytes;
      if (dey_store) de1 = (char *)dey_store + off;
      if (dcurl_store) dc1 = (char *)dcurl_store + off;
    }
    if (L.has_domain) {
      launch_fwd_h<T, ST>(L, s, cq, ey, hx, hz, m_ey_x, m_ey_z);
      launch_fwd_h<T, ST>(L, s, cq, dey, dhx, dhz, dm_ey_x, dm_ey_z);
    }
    const T *f0t = f0 ? f0 + t * fs : nullptr, *dft = df ? df + t * fs : nullptr;
    T *rt = r ? r + t * rs : nullptr, *bgt = background_r ? background_r + t * rs : nullptr;
    if (sr.stores(t) && sr.bf16) {
      using BF = __nv_bfloat16;
      launch_born_e<T, ST, BF>(L, s,
          L.g, ca, cb, dca, dcb, hx, hz, ey, m_hx_z, m_hz_x, dhx, dhz, dey, dm_hx_z, dm_hz_x,
          ps.src, ps.rec, f0t, dft, rt, bgt, (BF *)e1, (BF *)c1, (BF *)de1, (BF *)dc1, sh);
    } else {
      launch_born_e<T, ST, T>(L, s,
          L.g, ca, cb, dca, dcb, hx, hz, ey, m_hx_z, m_hz_x, dhx, dhz, dey, dm_hx_z, dm_hz_x,
          ps.src, ps.rec, f0t, dft, rt, bgt, (T *)e1, (T *)c1, (T *)de1, (T *)dc1, sh);
    }
    return sr.end(t, dst);
  };
  if (sr.host_side) {
    for (int64_t i = 0; i < nt; ++i)
      if (!step(i, st, nullptr, 0, false)) return;
  } else if (!run_step_blocks(nt, sr.want ? step_ratio : 1, st, prof, t_up, start_t, step)) {
    return;
  }
  count_launches(nt * (L.has_domain ? 3 : 1));
  if (TB_CUDA(cudaGetLastError())) return;
  sr.finish();
}

// Tangent (scattered-only) propagation from a stored device background
// history (cu_inst:1974-2086): step ratio 1, the history slot of step t at
// t * background_n_shots * ny * nx elements, scattered shot s reading
// background shot s % background_n_shots (direction batches).
template <typename T, int ST>
void tm_born_tangent_forward_with_storage(TIDE_TM_BORN_TANGENT_ARGS(T)) {
  (void)dt; (void)n_threads;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(step_ratio == 1,
             "TM2D born_tangent_forward_with_storage requires step_ratio=1, got %lld",
             (long long)step_ratio);
  TB_REQUIRE(nt >= 0 && start_t >= 0, "TM2D born_tangent_forward_with_storage: bad nt/start_t");
  TB_REQUIRE(ca && cb && cq && dca && dcb && dey && dhx && dhz && dm_ey_x && dm_ey_z &&
                 dm_hx_z && dm_hz_x && ey_store && curl_store,
             "TM2D born_tangent_forward_with_storage: a field, history or coefficient pointer "
             "is null");
  TB_REQUIRE(background_n_shots >= 1 && n_shots % background_n_shots == 0,
             "TM2D born_tangent_forward_with_storage: n_shots=%lld is not a multiple of "
             "background_n_shots=%lld", (long long)n_shots, (long long)background_n_shots);
  TB_REQUIRE(n_sources_per_shot == 0 || df,
             "TM2D born_tangent_forward_with_storage: sources without amplitudes");
  TB_REQUIRE(n_receivers_per_shot == 0 || r,
             "TM2D born_tangent_forward_with_storage: receivers without output");
  const bool bf16 = storage_format == 1;
  TB_REQUIRE(!bf16 || sizeof(T) == 4, "TM2D: bf16 snapshot storage requires float32 fields");
  Launch<T, ST> L;
  if (!make_launch(L, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, rdy, rdx, n_shots,
                   ny, nx, pml_y0, pml_x0, pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  cudaStream_t st = as_stream(compute_stream);
  PointScratch ps;
  L.narrow_e();
  if (!build_points(ps, L, L.e_tiles(),
                    sources_i, n_sources_per_shot, receivers_i, n_receivers_per_shot, st))
    return;
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  const int64_t bg_step = background_n_shots * ny * nx, sc_step = n_shots * ny * nx;
  ProfileScope prof(st);
  auto step = [&](int64_t i, cudaStream_t s, const int64_t *blk, int64_t B, bool) -> bool {
    const int64_t t = start_t + i;
    const StepShift sh{blk, B * fs, B * rs, B * sc_step, B * bg_step};
    if (L.has_domain) launch_fwd_h<T, ST>(L, s, cq, dey, dhx, dhz, dm_ey_x, dm_ey_z);
    const T *dft = df ? df + t * fs : nullptr;
    T *rt = r ? r + t * rs : nullptr;
    if (bf16) {
      using BF = __nv_bfloat16;
      launch_born_tangent_e<T, ST, BF>(L, s,
          L.g, ca, cb, dca, dcb, dhx, dhz, dey, dm_hx_z, dm_hz_x,
          (const BF *)ey_store + t * bg_step, (const BF *)curl_store + t * bg_step,
          (int)background_n_shots, ps.src, ps.rec, dft, rt,
          dey_store ? (BF *)dey_store + t * sc_step : nullptr,
          dcurl_store ? (BF *)dcurl_store + t * sc_step : nullptr, sh);
    } else {
      launch_born_tangent_e<T, ST, T>(L, s,
          L.g, ca, cb, dca, dcb, dhx, dhz, dey, dm_hx_z, dm_hz_x,
          (const T *)ey_store + t * bg_step, (const T *)curl_store + t * bg_step,
          (int)background_n_shots, ps.src, ps.rec, dft, rt,
          dey_store ? (T *)dey_store + t * sc_step : nullptr,
          dcurl_store ? (T *)dcurl_store + t * sc_step : nullptr, sh);
    }
    return true;
  };
  if (!run_step_blocks(nt, 1, st, prof, t_up, start_t, step)) return;
  count_launches(nt * (L.has_domain ? 2 : 1));
  TB_CUDA(cudaGetLastError());
}

// The CPML adjoint ping-pong buffers backward takes as adjoint_memory_scratch
// are allocated here in stream order (4 x n_shots x ny x nx).
template <typename T, int ST>
void tm_born_backward(TIDE_TM_BORN_BACKWARD_ARGS(T)) {
  (void)work_x; (void)work_z;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(n_shots >= 0 && ny > 0 && nx > 0, "TM2D born_backward: bad shape");
  cudaStream_t st = as_stream(compute_stream);
  T *scratch = nullptr;
  const size_t bytes = 4 * (size_t)n_shots * (size_t)ny * (size_t)nx * sizeof(T);
  if (TB_CUDA(pool_malloc((void **)&scratch, bytes > 0 ? bytes : sizeof(T), st))) return;
  tm_backward<T, ST>(ca, cb, cq, grad_r, lambda_ey, lambda_hx, lambda_hz, m_lambda_ey_x,
                     m_lambda_ey_z, m_lambda_hx_z, m_lambda_hz_x, scratch, ey_store_1,
                     ey_store_3, ey_filenames, curl_store_1, curl_store_3, curl_filenames,
                     grad_f, grad_ca, grad_cb, grad_ca_shot, grad_cb_shot, ay, by, ayh, byh, ax,
                     bx, axh, bxh, ky, kyh, kx, kxh, sources_i, receivers_i, rdy, rdx, dt, nt,
                     n_shots, ny, nx, n_sources_per_shot, n_receivers_per_shot, step_ratio,
                     storage_mode, storage_format, shot_bytes_uncomp, ca_requires_grad,
                     cb_requires_grad, ca_batched, cb_batched, cq_batched, start_t, pml_y0,
                     pml_x0, pml_y1, pml_x1, n_threads, device, compute_stream, storage_stream,
                     n_shots);
  TB_CUDA(cudaFreeAsync(scratch, st));
}

// ------------------------------------------- second-order Born adjoint
// Derivative of the scattered (and background) receivers in the background
// model, the perturbation and both source terms: the exact adjoint of the
// joint recurrence.  lam is the scattered state's adjoint (driven by grad_r),
// eta the background's (driven by grad_background_r and by the scattered
// update's dependence on the background, dEy' += dca Ey + dcb curlH).  Per
// step, with lam and eta at t+1: W = cb eta + dcb lam (the curl-H adjoint's
// source of the background) and eta_Ey <- ca eta + dca lam (k_bg_prep); the
// E- and H-phase adjoints of lam (cb, ca) and of eta (W in place of cb eta,
// unit ca); receivers and sources as two ordinary adjoints; at stored steps,
// step-major in this order: grad_ca += eta Ey + lam dEy, grad_cb += eta curl
// + lam dcurl, grad_dca += lam Ey, grad_dcb += lam curl (times k).

template <typename T>
__global__ void k_fill(T *__restrict__ p, int64_t n, T v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// W and the ca / dca part of eta_Ey on the update domain of every shot.
template <typename T>
__global__ void k_bg_prep(TMGeom<T> g, const T *__restrict__ ca, const T *__restrict__ cb,
                          const T *__restrict__ dca, const T *__restrict__ dcb,
                          const T *__restrict__ lam, T *__restrict__ eta, T *__restrict__ w,
                          int p) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int s = blockIdx.z;
  if (x < p || x >= g.nx - p + 1 || y < p || y >= g.ny - p + 1) return;
  const int64_t j = (int64_t)y * g.nx + x, i = (int64_t)s * g.N + j;
  const T cav = g.ca_b ? ca[i] : ca[j], dcav = g.ca_b ? dca[i] : dca[j];
  const T cbv = g.cb_b ? cb[i] : cb[j], dcbv = g.cb_b ? dcb[i] : dcb[j];
  const T l = lam[i], e = eta[i];
  w[i] = cbv * e + dcbv * l;
  eta[i] = cav * e + dcav * l;
}

// Step-major image of lam against the background history into the gradients
// of the perturbation: grad_dca[j] += sum_s lam Ey^t k, grad_dcb likewise
// with curl H^t (per shot when batched); snapshot shot s % bg_shots.
template <typename T, typename S>
__global__ void k_image_bg(TMGeom<T> g, const T *__restrict__ lam, const S *__restrict__ e_st,
                           const S *__restrict__ c_st, T *__restrict__ gdca,
                           T *__restrict__ gdcb, T kscale, int bg_shots, int p, StepShift sh) {
  if (sh.blk) {
    const int64_t jb = sh.block();
    e_st = shifted(e_st, sh.snap, jb);
    c_st = shifted(c_st, sh.snap, jb);
  }
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x < p || x >= g.nx - p + 1 || y < p || y >= g.ny - p + 1) return;
  const int64_t j = (int64_t)y * g.nx + x;
  T sa = 0, sb = 0;
  for (int s = 0; s < g.n_shots; ++s) {
    const int64_t i = (int64_t)s * g.N + j, k = (int64_t)(s % bg_shots) * g.N + j;
    const T v = lam[i];
    const T ta = v * Codec<S, T>::dec(e_st[k]) * kscale;
    const T tb = v * Codec<S, T>::dec(c_st[k]) * kscale;
    if (g.ca_b) gdca[i] = gdca[i] + ta;
    else sa = sa + ta;
    if (g.cb_b) gdcb[i] = gdcb[i] + tb;
    else sb = sb + tb;
  }
  if (!g.ca_b) gdca[j] = gdca[j] + sa;
  if (!g.cb_b) gdcb[j] = gdcb[j] + sb;
}

template <typename T, int ST>
void tm_born_backward_bggrad(TIDE_TM_BORN_BACKWARD_BGGRAD_ARGS(T)) {
  (void)f0; (void)df; (void)ey_store_3; (void)ey_filenames; (void)curl_store_3;
  (void)curl_filenames; (void)lambda_store; (void)eta_source_old; (void)work_eta_z;
  (void)grad_ca_shot; (void)grad_cb_shot; (void)grad_dca_shot; (void)grad_dcb_shot; (void)dt;
  (void)n_threads; (void)storage_stream;
  if (TB_CUDA(cudaSetDevice((int)device))) return;
  TB_REQUIRE(nt >= 0 && step_ratio >= 1 && start_t - nt >= 0,
             "TM2D born_backward_bggrad: bad nt/step_ratio/start_t");
  TB_REQUIRE(storage_mode == 0, "TM2D born_backward_bggrad: device storage mode only");
  TB_REQUIRE(ca_requires_grad && cb_requires_grad,
             "TM2D born_backward_bggrad: needs both the Ey and the curl H history");
  TB_REQUIRE(!capture_background_adjoint && !reuse_background_adjoint,
             "TM2D born_backward_bggrad: capturing or reusing the background adjoint is not "
             "built");
  TB_REQUIRE(ca && cb && cq && dca && dcb && ey && hx && hz && dey && dhx && dhz &&
                 m_lambda_ey_x && m_lambda_ey_z && m_lambda_hx_z && m_lambda_hz_x &&
                 m_eta_ey_x && m_eta_ey_z && m_eta_hx_z && m_eta_hz_x && work_eta_x &&
                 adjoint_memory_scratch && grad_ca && grad_cb && grad_dca && grad_dcb,
             "TM2D born_backward_bggrad: a field, memory, gradient or scratch pointer is null");
  TB_REQUIRE(ey_store_1 && curl_store_1 && dey_store && dcurl_store,
             "TM2D born_backward_bggrad: background and scattered histories are required");
  TB_REQUIRE(background_n_shots >= 1 && n_shots % background_n_shots == 0,
             "TM2D born_backward_bggrad: n_shots must be a multiple of background_n_shots");
  const bool bf16 = storage_format == 1;
  TB_REQUIRE(!bf16 || sizeof(T) == 4, "TM2D: bf16 snapshot storage requires float32 fields");
  const size_t esz = bf16 ? 2 : sizeof(T);
  TB_REQUIRE(shot_bytes_uncomp == ny * nx * (int64_t)esz,
             "TM2D born_backward_bggrad: shot_bytes_uncomp does not match ny*nx*elem");
  Launch<T, ST> L;
  if (!make_launch(L, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, rdy, rdx, n_shots,
                   ny, nx, pml_y0, pml_x0, pml_y1, pml_x1, ca_batched, cb_batched, cq_batched))
    return;
  if constexpr (ST == 2) pick_adj_h_rows<T, T>(L);
  L.narrow_e();
  cudaStream_t st = as_stream(compute_stream);
  const size_t SN = (size_t)n_shots * (size_t)L.g.N;
  const int bg = (int)background_n_shots;
  // the caller's adjoint state starts at zero (maxwell_tm_cuda_inst.cu:2963-2987)
  for (T *p : {ey, hx, hz, dey, dhx, dhz, m_lambda_ey_x, m_lambda_ey_z, m_lambda_hx_z,
               m_lambda_hz_x, m_eta_ey_x, m_eta_ey_z, m_eta_hx_z, m_eta_hz_x, work_eta_x})
    if (TB_CUDA(cudaMemsetAsync(p, 0, SN * sizeof(T), st))) return;
  if (TB_CUDA(cudaMemsetAsync(adjoint_memory_scratch, 0, 8 * SN * sizeof(T), st))) return;
  // unit coefficients standing for ca / cb in eta's phases (the kernels form
  // 1 * value exactly); per shot when the coefficients are batched
  T *ones = nullptr;
  const size_t n_ones = (ca_batched || cb_batched) ? SN : (size_t)L.g.N;
  if (TB_CUDA(pool_malloc((void **)&ones, n_ones * sizeof(T), st))) return;
  k_fill<T><<<592, 256, 0, st>>>(ones, (int64_t)n_ones, (T)1);
  PointScratch ps;
  if (!build_points(ps, L, L.ah_tiles(), sources_i, n_sources_per_shot, receivers_i,
                    n_receivers_per_shot, st))
    return;
  T *lc[4] = {m_lambda_ey_x, m_lambda_ey_z, m_lambda_hx_z, m_lambda_hz_x};
  T *ln[4], *ec[4] = {m_eta_ey_x, m_eta_ey_z, m_eta_hx_z, m_eta_hz_x}, *en[4];
  for (int m = 0; m < 4; ++m) {
    ln[m] = adjoint_memory_scratch + m * SN;
    en[m] = adjoint_memory_scratch + (4 + m) * SN;
  }
  T *w = work_eta_x;
  const int p = FD<ST>::P;
  const dim3 pblk(128, 1, 1), pgrid((unsigned)((nx + 127) / 128), (unsigned)ny, (unsigned)n_shots);
  const dim3 igrid((unsigned)((nx + 127) / 128), (unsigned)ny, 1);
  const int64_t fs = n_shots * n_sources_per_shot, rs = n_shots * n_receivers_per_shot;
  const size_t bstep = (size_t)shot_bytes_uncomp * (size_t)bg;       // background history step
  const size_t sstep = (size_t)shot_bytes_uncomp * (size_t)n_shots;  // scattered history step
  const int64_t bsnap = (int64_t)(bstep / esz), ssnap = (int64_t)(sstep / esz);
  int64_t launches = 1;
  ProfileScope prof(st);
  // step i of the call (time step start_t - 1 - i); the block pointers move
  // down (the adjoint walks the steps backwards)
  auto step = [&](int64_t i, cudaStream_t s, const int64_t *blk, int64_t B, bool) -> bool {
    const int64_t t = start_t - 1 - i;
    const int64_t qb = -(B / step_ratio);
    const StepShift sh_bg{blk, -B * fs, -B * rs, qb * bsnap, 0};
    const StepShift sh_sc{blk, -B * fs, -B * rs, qb * ssnap, 0};
    k_bg_prep<T><<<pgrid, pblk, 0, s>>>(L.g, ca, cb, dca, dcb, ey, dey, w, p);
    if (L.has_domain) {
      launch_adj_e<T, ST>(L, s, cb, ey, hx, hz, lc[2], lc[3], ln[2], ln[3]);
      launch_adj_e<T, ST>(L, s, ones, w, dhx, dhz, ec[2], ec[3], en[2], en[3]);
    }
    for (int m = 2; m < 4; ++m) {
      std::swap(lc[m], ln[m]);
      std::swap(ec[m], en[m]);
    }
    const bool grad_step = t % step_ratio == 0;
    const int64_t q = t / step_ratio;
    const char *es = grad_step ? (const char *)ey_store_1 + (size_t)q * bstep : nullptr;
    const char *cs = grad_step ? (const char *)curl_store_1 + (size_t)q * bstep : nullptr;
    const char *des = grad_step ? (const char *)dey_store + (size_t)q * sstep : nullptr;
    const char *dcs = grad_step ? (const char *)dcurl_store + (size_t)q * sstep : nullptr;
    const T *gbr = grad_background_r ? grad_background_r + t * rs : nullptr;
    const T *grt = grad_r ? grad_r + t * rs : nullptr;
    T *gf0 = grad_f0 ? grad_f0 + t * fs : nullptr;
    T *gdf = grad_df ? grad_df + t * fs : nullptr;
    auto both_h = [&](auto tag) {
      using SN_T = decltype(tag);
      GradArgs<T, SN_T> ge{(const SN_T *)es, (const SN_T *)cs, grad_ca, grad_cb,
                           (T)step_ratio, ca_batched, cb_batched, bg};
      launch_adj_h<T, ST, SN_T>(L, s, ones, cq, dhx, dhz, dey, ec[0], ec[1], en[0], en[1], ps,
                                gbr, gf0, ge, sh_bg);
      GradArgs<T, SN_T> gl{(const SN_T *)des, (const SN_T *)dcs, grad_ca, grad_cb,
                           (T)step_ratio, ca_batched, cb_batched, 0};
      launch_adj_h<T, ST, SN_T>(L, s, ca, cq, hx, hz, ey, lc[0], lc[1], ln[0], ln[1], ps, grt,
                                gdf, gl, sh_sc);
      if (grad_step)
        k_image_bg<T, SN_T><<<igrid, pblk, 0, s>>>(L.g, ey, (const SN_T *)es, (const SN_T *)cs,
                                                   grad_dca, grad_dcb, (T)step_ratio, bg, p,
                                                   sh_bg);
    };
    if (bf16) both_h(__nv_bfloat16(0.f));
    else both_h(T(0));
    for (int m = 0; m < 2; ++m) {
      std::swap(lc[m], ln[m]);
      std::swap(ec[m], en[m]);
    }
    return true;
  };
  if (!run_step_blocks(nt, step_ratio, st, prof, t_down, start_t, step)) return;
  // launches: 3 (+2 with a domain) per step and the image pass of each stored step
  for (int64_t t = start_t - 1; t >= start_t - nt; --t)
    launches += 3 + (L.has_domain ? 2 : 0) + (t % step_ratio == 0 ? 1 : 0);
  // leave the final memories in the caller's arrays
  const size_t nb = SN * sizeof(T);
  if (lc[0] != m_lambda_ey_x)
    for (int m = 0; m < 4; ++m) {
      T *dst[2] = {m == 0 ? m_lambda_ey_x : m == 1 ? m_lambda_ey_z : m == 2 ? m_lambda_hx_z
                                                                            : m_lambda_hz_x,
                   m == 0 ? m_eta_ey_x : m == 1 ? m_eta_ey_z : m == 2 ? m_eta_hx_z : m_eta_hz_x};
      if (TB_CUDA(cudaMemcpyAsync(dst[0], lc[m], nb, cudaMemcpyDeviceToDevice, st)) ||
          TB_CUDA(cudaMemcpyAsync(dst[1], ec[m], nb, cudaMemcpyDeviceToDevice, st)))
        return;
    }
  count_launches(launches);
  TB_CUDA(cudaFreeAsync(ones, st));
  TB_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace tb

#define TB_BORN_DEFINE(S, T)                                                           \
  extern "C" void maxwell_tm_##S##_##T##_born_forward_cuda(TIDE_TM_BORN_FORWARD_ARGS(T)) { \
    tb::tm_born_forward<T, S>(                                                         \
        ca, cb, cq, dca, dcb, f0, df, ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x, dey, dhx,   \
        dhz, dm_ey_x, dm_ey_z, dm_hx_z, dm_hz_x, r, background_r, ay, by, ayh, byh, ax, bx,   \
        axh, bxh, ky, kyh, kx, kxh, sources_i, receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx, \
        n_sources_per_shot, n_receivers_per_shot, step_ratio, ca_batched, cb_batched,         \
        cq_batched, start_t, pml_y0, pml_x0, pml_y1, pml_x1, n_threads, device,               \
        compute_stream);                                                               \
  }                                                                                    \
  extern "C" void maxwell_tm_##S##_##T##_born_forward_with_storage_cuda(              \
      TIDE_TM_BORN_FORWARD_WITH_STORAGE_ARGS(T)) {                                     \
    tb::tm_born_forward_with_storage<T, S>(                                            \
        ca, cb, cq, dca, dcb, f0, df, ey, hx, hz, m_ey_x, m_ey_z, m_hx_z, m_hz_x, dey, dhx,   \
        dhz, dm_ey_x, dm_ey_z, dm_hx_z, dm_hz_x, r, background_r, ey_store_1, ey_store_3,     \
        ey_filenames, curl_store_1, curl_store_3, curl_filenames, dey_store, dcurl_store, ay, \
        by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, sources_i, receivers_i, rdy, rdx,   \
        dt, nt, n_shots, ny, nx, n_sources_per_shot, n_receivers_per_shot, step_ratio,        \
        storage_mode, storage_format, shot_bytes_uncomp, ca_requires_grad, cb_requires_grad,  \
        ca_batched, cb_batched, cq_batched, start_t, pml_y0, pml_x0, pml_y1, pml_x1,          \
        n_threads, device, compute_stream, storage_stream);                            \
  }                                                                                    \
  extern "C" void maxwell_tm_##S##_##T##_born_tangent_forward_with_storage_cuda(      \
      TIDE_TM_BORN_TANGENT_ARGS(T)) {                                                  \
    tb::tm_born_tangent_forward_with_storage<T, S>(                                    \
        ca, cb, cq, dca, dcb, df, dey, dhx, dhz, dm_ey_x, dm_ey_z, dm_hx_z, dm_hz_x, r,       \
        ey_store, curl_store, dey_store, dcurl_store, ay, by, ayh, byh, ax, bx, axh, bxh, ky, \
        kyh, kx, kxh, sources_i, receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx,              \
        n_sources_per_shot, n_receivers_per_shot, step_ratio, storage_format,                 \
        background_n_shots, ca_batched, cb_batched, cq_batched, start_t, pml_y0, pml_x0,      \
        pml_y1, pml_x1, n_threads, device, compute_stream);                            \
  }                                                                                    \
  extern "C" void maxwell_tm_##S##_##T##_born_backward_cuda(TIDE_TM_BORN_BACKWARD_ARGS(T)) { \
    tb::tm_born_backward<T, S>(                                                        \
        ca, cb, cq, grad_r, lambda_ey, lambda_hx, lambda_hz, m_lambda_ey_x, m_lambda_ey_z,    \
        m_lambda_hx_z, m_lambda_hz_x, ey_store_1, ey_store_3, ey_filenames, curl_store_1,     \
        curl_store_3, curl_filenames, grad_f, grad_ca, grad_cb, grad_ca_shot, grad_cb_shot,   \
        work_x, work_z, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh, sources_i,      \
        receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx, n_sources_per_shot,                   \
        n_receivers_per_shot, step_ratio, storage_mode, storage_format, shot_bytes_uncomp,    \
        ca_requires_grad, cb_requires_grad, ca_batched, cb_batched, cq_batched, start_t,      \
        pml_y0, pml_x0, pml_y1, pml_x1, n_threads, device, compute_stream, storage_stream);  \
  }                                                                                    \
  extern "C" void maxwell_tm_##S##_##T##_born_backward_bggrad_cuda(                   \
      TIDE_TM_BORN_BACKWARD_BGGRAD_ARGS(T)) {                                          \
    tb::tm_born_backward_bggrad<T, S>(                                                 \
        ca, cb, cq, dca, dcb, f0, df, grad_r, grad_background_r, ey_store_1, ey_store_3,     \
        ey_filenames, curl_store_1, curl_store_3, curl_filenames, dey_store, dcurl_store,     \
        lambda_store, background_n_shots, ey, hx, hz, dey, dhx, dhz, grad_f0, grad_df,        \
        grad_ca, grad_cb, grad_dca, grad_dcb, m_lambda_ey_x, m_lambda_ey_z, m_lambda_hx_z,    \
        m_lambda_hz_x, m_eta_ey_x, m_eta_ey_z, m_eta_hx_z, m_eta_hz_x, eta_source_old,        \
        work_eta_x, work_eta_z, grad_ca_shot, grad_cb_shot, grad_dca_shot, grad_dcb_shot,     \
        adjoint_memory_scratch, ay, by, ayh, byh, ax, bx, axh, bxh, ky, kyh, kx, kxh,         \
        sources_i, receivers_i, rdy, rdx, dt, nt, n_shots, ny, nx, n_sources_per_shot,        \
        n_receivers_per_shot, step_ratio, storage_mode, storage_format, shot_bytes_uncomp,    \
        ca_requires_grad, cb_requires_grad, capture_background_adjoint,                       \
        reuse_background_adjoint, ca_batched, cb_batched, cq_batched, start_t, pml_y0,        \
        pml_x0, pml_y1, pml_x1, n_threads, device, compute_stream, storage_stream);           \
  }

TB_BORN_DEFINE(2, float)
TB_BORN_DEFINE(4, float)
TB_BORN_DEFINE(6, float)
TB_BORN_DEFINE(8, float)
TB_BORN_DEFINE(2, double)
TB_BORN_DEFINE(4, double)
TB_BORN_DEFINE(6, double)
TB_BORN_DEFINE(8, double)
