// Discrete adjoint of the 3-D Yee step (reverse-time sweep), sm_100a.
//
// The reference differentiates its 3-D FDTD with PyTorch autograd through
// every _time_step call (diffnano/solvers/fdtd3d.py:378-465); its
// "time_reversal" mode re-runs the forward with autograd in backward
// (_TimeReversalFDTD.backward, :166-219).  Here the transpose of one forward
// step is written out and run backwards in time, one launch per step.
//
// Forward step (dn_fdtd3d.cu, boundary rules folded into the coefficients):
//   H' = bH H + sum of (coef * forward differences of E)
//   E' = bE E + ce * curl,  curl = sum of (coef * backward differences of H')
// Reverse step, from the adjoint fields after the step (lE, lH) to the ones
// before it:
//   u_c = ce * lE_c                       (per E component)
//   lH' = lH + transpose(curl)(u)         needs u at the +1 neighbours
//   lE_prev = bE lE - transpose(H update)(lH')   needs lH' at the -1 neighbours
//   lH_prev = bH lH'
//   grad_ce += lE . curl                  (curl recorded by the forward replay)
// That is the forward kernel's data flow (H' needs E at +1, E' needs H' at
// -1), so this kernel reuses its z-march pipeline: the producer warp stages
// lEx, lEy, lEz, lHx, lHy, lHz, ce with a one-cell ring and the step's three
// curl arrays as tile boxes; each consumer warp owns two rows, recomputes lH'
// of the row above, takes x-1 neighbours by shuffle (lanes 0/1 compute the
// k0-1 halo column) and keeps the z-1 terms of the plane below in registers.
#include "dn_adjoint.cuh"
#include "dn_zmarch.cuh"

namespace dn {
namespace {

using namespace zm;

constexpr int NRING_A = 7;  // lEx lEy lEz lHx lHy lHz ce
constexpr int NTILE_A = 3;  // curl x y z of the step
constexpr int A_CE = 6;

template <typename T>
struct AdjCfg {
  static constexpr int S = sizeof(T) == 4 ? 4 : 3;
  static constexpr int MINB = sizeof(T) == 4 ? 2 : 1;
  using L = Layout<T, NRING_A, NTILE_A, S>;
};

template <typename T, int AXES>
__global__ void __launch_bounds__(NT, AdjCfg<T>::MINB)
    k_adj3d(const AdjParams<T> p, const __grid_constant__ TmapSet tm, const Plan plan) {
  using L = typename AdjCfg<T>::L;
  constexpr int S = L::S;
  constexpr int AE = L::RING_ARR / (int)sizeof(T);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const Smem<T, L> sm(smem_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int D = p.D, H = p.H, W = p.W;
  const long long py = p.py, pz = p.pz;
  const T dt = p.dt, idl = p.inv_dl;
  const Range R(plan, D);
  const int z0 = R.z0, z1 = R.z1, k0 = R.k0, j0 = R.j0;

  const int nj = pipe_setup(sm, R, D, H, W, p.b, p.c, p.status);
  if (nj == 0) return;

  if (warp == NCW) {
    const int slot = p.t - p.curl_t0;
    if (lane == 0)
      producer_run<T, L, NRING_A, NTILE_A>(sm, tm, R, nj, p.status,
                                           [slot](int) { return slot; });
    return;
  }

  volatile int* s_abort = sm.flags + 1;
  const int w = warp;
  const int ja = j0 + 2 * w;
  const int k = k0 + lane;
  const bool kin = k < W;
  const T dti = dt * idl;
  // coefficients of the forward step, boundary rules folded in (see
  // dn_fdtd3d.cu); "p1" = at the +1 neighbour along the named axis
  const T bK = sm.sbK[lane + 1], gK = sm.sgK[lane + 1];
  const T gKp1 = sm.sgK[lane + 2];  // column k+1
  const T bKh = sm.sbK[0], gKh = sm.sgK[0], gK0 = sm.sgK[1];  // columns k0-1, k0
  const T kf = (k < W - 1) ? T(1) : T(0);
  const T kb = (k > 0) ? T(1) : T(0);
  const T cKf = kf * dti * gK;     // forward x, H update
  const T cKb = kb * gK * idl;     // backward x, E update
  const T cKbp1 = gKp1 * idl;      // backward x at column k+1 (k+1 > 0)
  const T cKfh = dti * gKh;        // forward x at column k0-1 (k0-1 < W-1)
  const T cKbh = (k0 > 1) ? gKh * idl : T(0);  // backward x at column k0-1
  T bJ[4], gJ[4], cJf[4], cJb[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {  // rows ja-1 .. ja+2
    const int j = ja + r - 1;
    bJ[r] = sm.sbJ[2 * w + r];
    gJ[r] = sm.sgJ[2 * w + r];
    cJf[r] = (j < H - 1) ? dti * gJ[r] : T(0);
    cJb[r] = (j > 0) ? gJ[r] * idl : T(0);
  }
  // z-1 terms of rows ja, ja+1: vx_i = hx_c2 lHx', vy_i = hy_c1 lHy' of the plane below
  T pvxi[2] = {T(0), T(0)}, pvyi[2] = {T(0), T(0)};
  int q = 0;

  auto wait_full = [&](int qa) -> bool {
    const bool r = wait_phase(&sm.full[qa % S], (qa / S) & 1, s_abort);
    __syncwarp();
    return r;
  };
  auto release = [&](int qa) {
    __syncwarp();
    if (lane == 0) mbar_arrive(&sm.empty[qa % S]);
  };
  auto fail = [&]() {
    if (lane == 0) {
      report_status(p.status, DN_ETIMEOUT);
      *s_abort = 1;
    }
  };
  // per-plane coefficients of the z roles: e_ci (E update, backward z, scale
  // only; the i>0 rule is applied by the caller), hx_c2 / hy_c1 (H update,
  // forward z), hy_b, bI
  auto i_roles = [&](int i, T& e_ci, T& hx_c2, T& hy_c1, T& hy_b, T& bI) {
    if (AXES == DN_AXES_REFERENCE) {
      e_ci = gK * idl;
      hx_c2 = dti * gK;
      hy_c1 = dti * gK;
      hy_b = bK;
      bI = T(1);
    } else {
      bI = static_cast<T>(__ldg(p.b[0] + i));
      const T gI = static_cast<T>(1.0 + __ldg(p.c[0] + i));
      e_ci = gI * idl;
      hx_c2 = dti * gI;
      hy_c1 = dti * gI;
      hy_b = bI;
    }
  };
  auto e_ci_at = [&](int i) -> T {  // e_ci of plane i (i < D)
    if (AXES == DN_AXES_REFERENCE) return gK * idl;
    return static_cast<T>(1.0 + __ldg(p.c[0] + i)) * idl;
  };

  // lH' (all three) at row r (0..2) of this lane's column.  cur/nxt point at
  // row ja-1, column k of the plane's / next plane's stage; fi_next is 0 on
  // the last plane (no +z neighbour) and fi_prev is 0 on the first (no E-update
  // z term there).
  auto lam_h = [&](const T* cur, const T* nxt, int r, T e_ci, T e_ci_n, T fi_prev, T fi_next,
                   T& lhx, T& lhy, T& lhz) {
    const int e = r * BX;
    const T ce = cur[A_CE * AE + e];
    const T ux = ce * cur[DN_EX * AE + e], uy = ce * cur[DN_EY * AE + e],
            uz = ce * cur[DN_EZ * AE + e];
    const T ce_j = cur[A_CE * AE + e + BX];
    const T ux_j = ce_j * cur[DN_EX * AE + e + BX], uz_j = ce_j * cur[DN_EZ * AE + e + BX];
    const T ce_k = cur[A_CE * AE + e + 1];
    const T uy_k = ce_k * cur[DN_EY * AE + e + 1], uz_k = ce_k * cur[DN_EZ * AE + e + 1];
    const T ce_i = nxt[A_CE * AE + e];
    const T ux_i = ce_i * nxt[DN_EX * AE + e], uy_i = ce_i * nxt[DN_EY * AE + e];
    const T eci = e_ci * fi_prev, ecin = e_ci_n * fi_next;
    const T eyc2 = AXES == DN_AXES_REFERENCE ? kb * gJ[r] * idl : cKb;
    const T eyc2p1 = AXES == DN_AXES_REFERENCE ? gJ[r] * idl : cKbp1;
    lhx = cur[DN_HX * AE + e] + (eci * uy - ecin * uy_i) - (cJb[r] * uz - cJb[r + 1] * uz_j);
    lhy = cur[DN_HY * AE + e] - (eci * ux - ecin * ux_i) + (cKb * uz - cKbp1 * uz_k);
    lhz = cur[DN_HZ * AE + e] + (cJb[r] * ux - cJb[r + 1] * ux_j) - (eyc2 * uy - eyc2p1 * uy_k);
  };

  // ---- warm-up: z-1 terms from plane z0-1 ------------------------------------
  if (z0 > 0) {
    if (!(wait_full(q) && wait_full(q + 1))) {
      fail();
      return;
    }
    const int i = z0 - 1;
    T e_ci, hx_c2, hy_c1, hy_b, bI;
    i_roles(i, e_ci, hx_c2, hy_c1, hy_b, bI);
    const T e_ci_n = e_ci_at(i + 1);
    const T* cur = sm.arr(q, 0) + 2 * w * BX + lane + 4;
    const T* nxt = sm.arr(q + 1, 0) + 2 * w * BX + lane + 4;
#pragma unroll
    for (int r = 1; r < 3; ++r) {
      T lhx, lhy, lhz;
      lam_h(cur, nxt, r, e_ci, e_ci_n, i > 0 ? T(1) : T(0), T(1), lhx, lhy, lhz);
      pvxi[r - 1] = hx_c2 * lhx;  // i < D-1 here
      pvyi[r - 1] = hy_c1 * lhy;
    }
    release(q);
    ++q;
  }

  // ---- march -----------------------------------------------------------------
  for (int i = z0; i < z1; ++i) {
    const bool has_next = (i + 1 < D);
    if ((i == 0 && !wait_full(q)) || (has_next && !wait_full(q + 1))) {
      fail();
      return;
    }
    T e_ci, hx_c2, hy_c1, hy_b, bI;
    i_roles(i, e_ci, hx_c2, hy_c1, hy_b, bI);
    const T e_ci_n = has_next ? e_ci_at(i + 1) : T(0);
    const T fi_prev = i > 0 ? T(1) : T(0);
    const T fi_next = has_next ? T(1) : T(0);
    const T* cur = sm.arr(q, 0) + 2 * w * BX + lane + 4;
    const T* nxt = has_next ? sm.arr(q + 1, 0) + 2 * w * BX + lane + 4 : cur;
    // issue the FP64 gradient loads now; they are consumed after lH'
    const long long o_plane = i * pz + (long long)ja * py + k;
    double gpre[2];
#pragma unroll
    for (int r = 1; r < 3; ++r)
      gpre[r - 1] = (ja + r - 1 < H && kin) ? p.grad[o_plane + (r - 1) * py] : 0.0;

    // ---- lH' of rows ja-1, ja, ja+1 --------------------------------------
    T LHx[3], LHy[3], LHz[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
      lam_h(cur, nxt, r, e_ci, e_ci_n, fi_prev, fi_next, LHx[r], LHy[r], LHz[r]);

    // ---- k0-1 halo column: lHy', lHz' of rows ja, ja+1 (lanes 0, 1) -------
    // v_k terms there: vy_k = hy_c2 lHy', vz_k = cKf lHz'
    T hvyk = T(0), hvzk = T(0);
    if (lane < 2 && k0 > 0) {
      const int r = 1 + lane;
      const T gJr = lane == 0 ? gJ[1] : gJ[2];
      const T cJbr = lane == 0 ? cJb[1] : cJb[2];
      const T cJbr1 = lane == 0 ? cJb[2] : cJb[3];
      const int e = r * BX - 1 - lane;  // column k0-1 (pointers sit at k0+lane)
      const T ce = cur[A_CE * AE + e];
      const T ux = ce * cur[DN_EX * AE + e], uy = ce * cur[DN_EY * AE + e],
              uz = ce * cur[DN_EZ * AE + e];
      const T ce_j = cur[A_CE * AE + e + BX];
      const T ux_j = ce_j * cur[DN_EX * AE + e + BX];
      const T ce_k = cur[A_CE * AE + e + 1];
      const T uy_k = ce_k * cur[DN_EY * AE + e + 1], uz_k = ce_k * cur[DN_EZ * AE + e + 1];
      const T ce_i = nxt[A_CE * AE + e];
      const T ux_i = ce_i * nxt[DN_EX * AE + e];
      const T eci = (AXES == DN_AXES_REFERENCE ? gKh * idl : e_ci) * fi_prev;
      const T ecin = (AXES == DN_AXES_REFERENCE ? gKh * idl : e_ci_n) * fi_next;
      const T cKb0 = gK0 * idl;  // backward x at column k0 (> 0)
      const T eyc2 = AXES == DN_AXES_REFERENCE ? (k0 > 1 ? gJr * idl : T(0)) : cKbh;
      const T eyc2p1 = AXES == DN_AXES_REFERENCE ? gJr * idl : cKb0;
      const T lhy = cur[DN_HY * AE + e] - (eci * ux - ecin * ux_i) + (cKbh * uz - cKb0 * uz_k);
      const T lhz = cur[DN_HZ * AE + e] + (cJbr * ux - cJbr1 * ux_j) - (eyc2 * uy - eyc2p1 * uy_k);
      const T hyc2 = AXES == DN_AXES_REFERENCE ? dti * gJr : cKfh;
      hvyk = hyc2 * lhy;
      hvzk = cKfh * lhz;
    }
    const T hvyk0 = __shfl_sync(FULL_MASK, hvyk, 0), hvyk1 = __shfl_sync(FULL_MASK, hvyk, 1);
    const T hvzk0 = __shfl_sync(FULL_MASK, hvzk, 0), hvzk1 = __shfl_sync(FULL_MASK, hvzk, 1);

    // ---- previous adjoint fields of rows ja, ja+1 ---------------------------
    const T* ct = sm.tile_arr(q, NRING_A, 0) + (2 * w) * TX + lane;
    constexpr int TE = L::TILE_ARR / (int)sizeof(T);
#pragma unroll
    for (int r = 1; r < 3; ++r) {
      const int j = ja + r - 1;
      const T hyc2 = AXES == DN_AXES_REFERENCE ? kf * dti * gJ[r] : cKf;
      // v terms of this lane
      const T vxj = cJf[r] * LHx[r], vzj = cJf[r] * LHz[r];
      const T vxi = has_next ? hx_c2 * LHx[r] : T(0);
      const T vyi = has_next ? hy_c1 * LHy[r] : T(0);
      const T vyk = hyc2 * LHy[r], vzk = cKf * LHz[r];
      // -1 neighbours
      const T vxj_m = cJf[r - 1] * LHx[r - 1], vzj_m = cJf[r - 1] * LHz[r - 1];
      T vyk_m = __shfl_up_sync(FULL_MASK, vyk, 1);
      T vzk_m = __shfl_up_sync(FULL_MASK, vzk, 1);
      if (lane == 0) {
        vyk_m = r == 1 ? hvyk0 : hvyk1;
        vzk_m = r == 1 ? hvzk0 : hvzk1;
      }
      if (j < H && kin) {
        const int e = r * BX;
        const T lex = cur[DN_EX * AE + e], ley = cur[DN_EY * AE + e], lez = cur[DN_EZ * AE + e];
        const T ex_b = AXES == DN_AXES_REFERENCE ? bJ[r] * bK : bJ[r] * bI;
        const T ey_b = AXES == DN_AXES_REFERENCE ? bK * bJ[r] : bI * bK;
        const T ez_b = bK * bJ[r];
        const T nlex = ex_b * lex + (vyi - pvyi[r - 1]) - (vzj - vzj_m);
        const T nley = ey_b * ley - (vxi - pvxi[r - 1]) + (vzk - vzk_m);
        const T nlez = ez_b * lez + (vxj - vxj_m) - (vyk - vyk_m);
        const long long o = o_plane + (r - 1) * py;
        const int et = (r - 1) * TX;
        const double gsum = static_cast<double>(lex) * static_cast<double>(ct[et]) +
                            static_cast<double>(ley) * static_cast<double>(ct[TE + et]) +
                            static_cast<double>(lez) * static_cast<double>(ct[2 * TE + et]);
        p.grad[o] = gpre[r - 1] + gsum;
        p.out[DN_EX][o] = nlex;
        p.out[DN_EY][o] = nley;
        p.out[DN_EZ][o] = nlez;
        p.out[DN_HX][o] = bJ[r] * LHx[r];
        p.out[DN_HY][o] = hy_b * LHy[r];
        p.out[DN_HZ][o] = bK * LHz[r];
      }
      pvxi[r - 1] = vxi;
      pvyi[r - 1] = vyi;
    }
    release(q);
    ++q;
  }
  if (z1 < D) release(q);
}

template <typename T, int AXES>
int launch_adj(AdjParams<T> p, void* const la[6], void* const lb[6], const dn_grid* g,
               const dn_curl_record* curl, const dn_monitor* mons, int n_mon, int t_end,
               int nsteps, cudaStream_t s) {
  using L = typename AdjCfg<T>::L;
  int rc;
  TmapSet ta, tb;
  for (int c = 0; c < 6; ++c) {
    if ((rc = encode_ring(&ta.m[c], la[c], g, sizeof(T))) != DN_OK) return rc;
    if ((rc = encode_ring(&tb.m[c], lb[c], g, sizeof(T))) != DN_OK) return rc;
  }
  if ((rc = encode_ring(&ta.m[A_CE], p.ce, g, sizeof(T))) != DN_OK) return rc;
  tb.m[A_CE] = ta.m[A_CE];
  for (int c = 0; c < 3; ++c) {
    if ((rc = encode_tile4(&ta.m[NRING_A + c], curl->curl[c], g, sizeof(T), curl->nslots,
                           curl->step_stride)) != DN_OK)
      return rc;
    tb.m[NRING_A + c] = ta.m[NRING_A + c];
  }
  int dev = 0, nsm = 0;
  DN_CUDA_CHECK(cudaGetDevice(&dev));
  DN_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  long long nctas = 0;
  const Plan plan = make_plan(g, (long long)nsm * AdjCfg<T>::MINB, &nctas);
  if (nctas > 0x7fffffffLL) return DN_EUNSUPPORTED;
  const size_t smem = L::BYTES;
  if (smem > 227 * 1024) return DN_EUNSUPPORTED;
  auto kern = k_adj3d<T, AXES>;
  DN_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
  for (int n = 0; n < nsteps; ++n) {
    const bool even = (n % 2) == 0;
    for (int c = 0; c < 6; ++c) {
      p.in[c] = static_cast<const T*>(even ? la[c] : lb[c]);
      p.out[c] = static_cast<T*>(even ? lb[c] : la[c]);
    }
    p.t = t_end - 1 - n;
    if (n_mon > 0 && (rc = inject_monitors<T>(p, mons, n_mon, true, 0, s)) != DN_OK) return rc;
    kern<<<(unsigned)nctas, NT, smem, s>>>(p, even ? ta : tb, plan);
  }
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

template <typename T>
int adjoint3d(const dn_grid* g, void* const la[6], void* const lb[6], const void* ce,
              const dn_cpml* cpml, const dn_curl_record* curl, double* grad,
              const dn_monitor* mons, int32_t n_mon, int32_t t_end, int32_t nsteps,
              int32_t* status, void* stream, int32_t* final_in_b) {
  AdjParams<T> p;
  int rc = build_adj_params<T>(true, g, la, lb, ce, cpml, curl, grad, t_end, nsteps, status, &p);
  if (rc != DN_OK) return rc;
  if (!final_in_b || n_mon < 0 || n_mon > DN_MAX_MONITORS || (n_mon > 0 && !mons))
    return DN_EINVAL;
  if (!mons_steps_ok(mons, n_mon, (int64_t)t_end - nsteps, t_end)) return DN_EINVAL;
  const void* ptrs[16];
  for (int c = 0; c < 6; ++c) {
    ptrs[c] = la[c];
    ptrs[6 + c] = lb[c];
  }
  ptrs[12] = ce;
  for (int c = 0; c < 3; ++c) ptrs[13 + c] = curl->curl[c];
  if (!tma_ok(g, sizeof(T), ptrs, 16) || (curl->step_stride * (int64_t)sizeof(T)) % 16)
    return DN_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  rc = g->axes == DN_AXES_REFERENCE
           ? launch_adj<T, DN_AXES_REFERENCE>(p, la, lb, g, curl, mons, n_mon, t_end, nsteps, s)
           : launch_adj<T, DN_AXES_PHYSICAL>(p, la, lb, g, curl, mons, n_mon, t_end, nsteps, s);
  if (rc != DN_OK) return rc;
  *final_in_b = nsteps % 2;
  return DN_OK;
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_fdtd3d_adjoint(const dn_grid* g, void* const la[6], void* const lb[6],
                                     const void* ce, const dn_cpml* cpml,
                                     const dn_curl_record* curl, double* grad_ce,
                                     const dn_monitor* mons, int32_t n_mon, int32_t t_end,
                                     int32_t nsteps, int32_t* status, void* stream,
                                     int32_t* final_in_b) {
  if (!g) return DN_EINVAL;
  if (g->dtype == DN_F32)
    return dn::adjoint3d<float>(g, la, lb, ce, cpml, curl, grad_ce, mons, n_mon, t_end, nsteps,
                                status, stream, final_in_b);
  if (g->dtype == DN_F64)
    return dn::adjoint3d<double>(g, la, lb, ce, cpml, curl, grad_ce, mons, n_mon, t_end, nsteps,
                                 status, stream, final_in_b);
  return DN_EINVAL;
}
