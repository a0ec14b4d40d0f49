// Discrete adjoint of the 2-D TMz / TE step (reverse-time sweep), sm_100a.
//
// The reference differentiates its FDTD with PyTorch autograd through every
// _time_step_tm / _time_step_te call (diffnano/solvers/fdtd2d.py:233-303).
// Here the transpose of one step is written out by hand and run backwards in
// time, one launch per step, from adjoint fields lambda (the gradient of the
// loss with respect to the fields after the step) to the adjoint fields
// before it, while dL/d(dt/eps) accumulates in FP64.
//
// With the forward step written as (TM; mu-coefficients c = (1+c_prof)/dl)
//   Hx' = by Hx - dt cy dEz/dj          Hy' = bx Hy + dt cx dEz/di
//   Ez' = bx by Ez + ce (cx dHy'/di - cy dHx'/dj)         (ce = dt/eps)
// the reverse step is
//   u = ce * lambda_Ez
//   lHx' = lHx - cy (u - u(j+1)) [j>0 weight on u]   lHy' = lHy + cx (u - u(i+1))
//   lEz_prev = bx by lEz + (vx - vx(j-1)) - (vy - vy(i-1)),  vx = dt cy lHx', vy = dt cx lHy'
//   lHx_prev = by lHx',  lHy_prev = bx lHy',  grad_ce += lEz * curl_z
// with the same boundary rules as the forward differences (a coefficient is
// zero where the forward difference is).  TE is the mirror image: the adjoint
// of the Hz update comes first, then the E updates.
//
// Work layout (the forward step's): a warp owns a strip of 32*VEC columns,
// VEC adjacent columns per lane with 16-byte loads and stores when rows and
// arrays are 16-byte aligned, and R consecutive rows, which it marches down
// with the row neighbours in registers and the column neighbours from its own
// registers or the adjacent lane (shuffle).  The edge lanes load or recompute
// the one value outside the strip (TM: vx at column j0-1, u at j0+32*VEC;
// TE: lambda_Hz at j0-1, ux at j0+32*VEC) and the warp recomputes the
// intermediate row above (TM: vy) or below (TE: lambda_E', uy) its own, with
// the owner's arithmetic: no shared memory, no barrier; ping-pong buffers.
#include <algorithm>
#include <atomic>

#include "dn_adjoint.cuh"
#include "dn_strip.cuh"

namespace dn {
namespace {

constexpr int NTA = 256;  // 8 warps stacked along the rows
constexpr int WARPS_A = NTA / 32;
constexpr unsigned FULL_A = STRIP_FULL_MASK;

// TM reverse step, rows [ia, ib) of the strip of columns from j0.
template <typename T, int VEC>
__device__ __forceinline__ void adj_march_tm(const AdjParams<T>& p, int j0, int ia, int ib) {
  using V = Vec<T, VEC>;
  const int lane = threadIdx.x & 31;
  const int H = p.H, W = p.W;
  const long long py = p.py;
  const int jv = j0 + lane * VEC;
  const bool any = jv < W, full = jv + VEC <= W;
  const T dt = p.dt, idl = p.inv_dl;
  const T* lEz = p.in[DN_EZ];
  const T* lHx = p.in[DN_HX];
  const T* lHy = p.in[DN_HY];
  const long long cslot = (long long)(p.t - p.curl_t0) * p.curl_stride;
  V bx, gx;  // gx = (1 + c_x) / dl
#pragma unroll
  for (int q = 0; q < VEC; ++q) {
    const int j = jv + q;
    bx[q] = j < W ? static_cast<T>(p.b[2][j]) : T(1);
    gx[q] = (j < W ? static_cast<T>(1.0 + p.c[2][j]) : T(1)) * idl;
  }
  const bool edge_l = lane == 0 && j0 > 0;         // recomputes vx at column j0-1
  const bool edge_r = lane == 31 && jv + VEC < W;  // loads u at column j0+32*VEC

  long long o = (long long)ia * py + jv;
  V lez_c = ldv<T, VEC>(lEz, o, any, full, jv, W);
  V u_c;
  {
    const V ce = ldv<T, VEC>(p.ce, o, any, full, jv, W);
#pragma unroll
    for (int q = 0; q < VEC; ++q) u_c[q] = ce[q] * lez_c[q];
  }
  // vy of row ia-1, recomputed with its owner's arithmetic (row ia-1 < H-1)
  V vy_up;
#pragma unroll
  for (int q = 0; q < VEC; ++q) vy_up[q] = T(0);
  if (ia > 0) {
    const V lez_u = ldv<T, VEC>(lEz, o - py, any, full, jv, W);
    const V ce_u = ldv<T, VEC>(p.ce, o - py, any, full, jv, W);
    const V lhy_u = ldv<T, VEC>(lHy, o - py, any, full, jv, W);
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const T uu = ce_u[q] * lez_u[q];
      const T lh = lhy_u[q] + gx[q] * ((ia - 1 > 0 ? uu : T(0)) - u_c[q]);
      vy_up[q] = dt * gx[q] * lh;
    }
  }
  for (int i = ia; i < ib; ++i, o += py) {
    const bool nxt = i + 1 < H;
    const V lez_n = ldv<T, VEC>(lEz, o + py, any && nxt, full, jv, W);
    const V ce_n = ldv<T, VEC>(p.ce, o + py, any && nxt, full, jv, W);
    const V lhx = ldv<T, VEC>(lHx, o, any, full, jv, W);
    const V lhy = ldv<T, VEC>(lHy, o, any, full, jv, W);
    const V crl = ldv<T, VEC>(p.curl[2], cslot + o, any, full, jv, W);
    Vec<double, VEC> g = ldv<double, VEC, LD_PLAIN>(p.grad, o, any, full, jv, W);
    const T ce_r31 = ld(p.ce, o + VEC, edge_r), lez_r31 = ld(lEz, o + VEC, edge_r);
    const T ce_l0 = ld(p.ce, o - 1, edge_l), lez_l0 = ld(lEz, o - 1, edge_l);
    const T lhx_l0 = ld(lHx, o - 1, edge_l);
    const T by = static_cast<T>(p.b[1][i]);
    const T gy = static_cast<T>(1.0 + p.c[1][i]) * idl;

    V u_n;
#pragma unroll
    for (int q = 0; q < VEC; ++q) u_n[q] = ce_n[q] * lez_n[q];
    T u_rl = __shfl_down_sync(FULL_A, u_c[0], 1);
    if (lane == 31) u_rl = ce_r31 * lez_r31;
    V a, b, vx, vy;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      const T u_r = (q < VEC - 1) ? u_c[q < VEC - 1 ? q + 1 : q] : u_rl;
      a[q] = lhx[q] - gy * ((j > 0 ? u_c[q] : T(0)) - u_r);
      b[q] = lhy[q] + gx[q] * ((i > 0 ? u_c[q] : T(0)) - u_n[q]);
      vx[q] = (j < W - 1) ? dt * gy * a[q] : T(0);
      vy[q] = (i < H - 1) ? dt * gx[q] * b[q] : T(0);
    }
    T vx_ll = __shfl_up_sync(FULL_A, vx[VEC - 1], 1);
    if (lane == 0) {
      T v = T(0);
      if (edge_l) {  // column j0-1 < W-1
        const T ul = ce_l0 * lez_l0;
        const T lh = lhx_l0 - gy * ((j0 - 1 > 0 ? ul : T(0)) - u_c[0]);
        v = dt * gy * lh;
      }
      vx_ll = v;
    }
    V lez_p, lhx_p, lhy_p;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const T vx_l = (q > 0) ? vx[q > 0 ? q - 1 : 0] : vx_ll;
      g[q] += static_cast<double>(lez_c[q]) * static_cast<double>(crl[q]);
      lez_p[q] = bx[q] * by * lez_c[q] + (vx[q] - vx_l) - (vy[q] - vy_up[q]);
      lhx_p[q] = by * a[q];
      lhy_p[q] = bx[q] * b[q];
    }
    if (any) {
      stv(p.grad, o, g, full, jv, W);
      stv(p.out[DN_EZ], o, lez_p, full, jv, W);
      stv(p.out[DN_HX], o, lhx_p, full, jv, W);
      stv(p.out[DN_HY], o, lhy_p, full, jv, W);
    }
    vy_up = vy;
    u_c = u_n;
    lez_c = lez_n;
  }
}

// TE reverse step, rows [ia, ib) of the strip of columns from j0.  The
// E-adjoint half of row i+1 (lambda_E', ux, uy) is computed in iteration i,
// since the Hz-adjoint of row i needs uy of row i+1, and carried to i+1; each
// row's gradient is accumulated once, by the warp that owns the row.
template <typename T, int VEC>
__device__ __forceinline__ void adj_march_te(const AdjParams<T>& p, int j0, int ia, int ib) {
  using V = Vec<T, VEC>;
  const int lane = threadIdx.x & 31;
  const int H = p.H, W = p.W;
  const long long py = p.py;
  const int jv = j0 + lane * VEC;
  const bool any = jv < W, full = jv + VEC <= W;
  const T dt = p.dt, idl = p.inv_dl;
  const T* lHz = p.in[DN_HZ];
  const T* lEx = p.in[DN_EX];
  const T* lEy = p.in[DN_EY];
  const long long cslot = (long long)(p.t - p.curl_t0) * p.curl_stride;
  V bx, gxr, cx;  // gxr = 1 + c_x, cx = dt (1 + c_x) / dl
#pragma unroll
  for (int q = 0; q < VEC; ++q) {
    const int j = jv + q;
    bx[q] = j < W ? static_cast<T>(p.b[2][j]) : T(1);
    gxr[q] = j < W ? static_cast<T>(1.0 + p.c[2][j]) : T(1);
    cx[q] = dt * gxr[q] * idl;
  }
  const bool edge_l = lane == 0 && j0 > 0;         // loads lambda_Hz at column j0-1
  const bool edge_r = lane == 31 && jv + VEC < W;  // recomputes ux at column j0+32*VEC
  const T gxr_r = edge_r ? static_cast<T>(1.0 + p.c[2][jv + VEC]) : T(1);

  // E-adjoint half of row r (offset oo) from lambda_Hz of rows r (lh) and
  // r-1 (lh_u); accumulates the row's gradient when `own`; all 32 lanes call it
  auto e_row = [&](int r, long long oo, const V& lh, const V& lh_u, bool own, V& a, V& b, V& ux,
                   V& uy) {
    const V lex = ldv<T, VEC>(lEx, oo, any, full, jv, W);
    const V ley = ldv<T, VEC>(lEy, oo, any, full, jv, W);
    const V ce = ldv<T, VEC>(p.ce, oo, any, full, jv, W);
    const T lh_l0 = ld(lHz, oo - 1, edge_l);
    const T gyr = static_cast<T>(1.0 + p.c[1][r]);
    const T cy = dt * gyr * idl;
    T lh_ll = __shfl_up_sync(FULL_A, lh[VEC - 1], 1);
    if (lane == 0) lh_ll = lh_l0;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int j = jv + q;
      const T lh_l = (q > 0) ? lh[q > 0 ? q - 1 : 0] : lh_ll;
      const T wj = (j < W - 1) ? cy * lh[q] : T(0);
      const T wjm = (j > 0) ? cy * lh_l : T(0);
      const T wi = (r < H - 1) ? cx[q] * lh[q] : T(0);
      const T wim = (r > 0) ? cx[q] * lh_u[q] : T(0);
      a[q] = lex[q] + wj - wjm;
      b[q] = ley[q] - wi + wim;
      ux[q] = (j > 0) ? ce[q] * gxr[q] * idl * a[q] : T(0);
      uy[q] = (r > 0) ? ce[q] * gyr * idl * b[q] : T(0);
    }
    if (own && any) {
      const V c0 = ldv<T, VEC>(p.curl[0], cslot + oo, any, full, jv, W);
      const V c1 = ldv<T, VEC>(p.curl[1], cslot + oo, any, full, jv, W);
      Vec<double, VEC> g = ldv<double, VEC, LD_PLAIN>(p.grad, oo, any, full, jv, W);
#pragma unroll
      for (int q = 0; q < VEC; ++q)
        g[q] += static_cast<double>(a[q]) * static_cast<double>(c0[q]) +
                static_cast<double>(b[q]) * static_cast<double>(c1[q]);
      stv(p.grad, oo, g, full, jv, W);
    }
  };

  long long o = (long long)ia * py + jv;
  V lh_c = ldv<T, VEC>(lHz, o, any, full, jv, W);
  const V lh_u = ldv<T, VEC>(lHz, o - py, any && ia > 0, full, jv, W);
  V a_c, b_c, ux_c, uy_c;
  e_row(ia, o, lh_c, lh_u, true, a_c, b_c, ux_c, uy_c);
  for (int i = ia; i < ib; ++i, o += py) {
    const bool nxt = i + 1 < H;
    const V lh_n = ldv<T, VEC>(lHz, o + py, any && nxt, full, jv, W);
    const T lex31 = ld(lEx, o + VEC, edge_r), ce31 = ld(p.ce, o + VEC, edge_r);
    const T lh31 = ld(lHz, o + VEC, edge_r);
    const T by = static_cast<T>(p.b[1][i]);
    const T cy = dt * static_cast<T>(1.0 + p.c[1][i]) * idl;
    V a_n, b_n, ux_n, uy_n;
#pragma unroll
    for (int q = 0; q < VEC; ++q) a_n[q] = b_n[q] = ux_n[q] = uy_n[q] = T(0);
    if (nxt) e_row(i + 1, o + py, lh_n, lh_c, i + 1 < ib, a_n, b_n, ux_n, uy_n);

    T ux_rl = __shfl_down_sync(FULL_A, ux_c[0], 1);
    if (lane == 31) {
      T v = T(0);
      if (edge_r) {  // column jh = j0+32*VEC > 0
        const T wj = (jv + VEC < W - 1) ? cy * lh31 : T(0);
        const T wjm = cy * lh_c[VEC - 1];
        const T lex_p = lex31 + wj - wjm;
        v = ce31 * gxr_r * idl * lex_p;
      }
      ux_rl = v;
    }
    V lhz_p, lex_p, ley_p;
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const T ux_r = (q < VEC - 1) ? ux_c[q < VEC - 1 ? q + 1 : q] : ux_rl;
      lhz_p[q] = bx[q] * by * lh_c[q] + (ux_c[q] - ux_r) - (uy_c[q] - uy_n[q]);
      lex_p[q] = bx[q] * a_c[q];
      ley_p[q] = by * b_c[q];
    }
    if (any) {
      stv(p.out[DN_HZ], o, lhz_p, full, jv, W);
      stv(p.out[DN_EX], o, lex_p, full, jv, W);
      stv(p.out[DN_EY], o, ley_p, full, jv, W);
    }
    lh_c = lh_n;
    a_c = a_n;
    b_c = b_n;
    ux_c = ux_n;
    uy_c = uy_n;
  }
}

template <typename T, int POL, int VEC>
__global__ void __launch_bounds__(NTA, 2) k_adj2d(const AdjParams<T> p, int R) {
  // a previous launch that recorded an error turns this one into a no-op
  if (p.status != nullptr && *reinterpret_cast<volatile int*>(p.status) != 0) return;
  const int warp = threadIdx.x >> 5;
  const int j0 = blockIdx.x * 32 * VEC;
  const long long ia = ((long long)blockIdx.y * WARPS_A + warp) * R;
  if (ia >= p.H) return;  // whole warp: the shuffles see all 32 lanes
  const int ib = static_cast<int>(std::min<long long>(ia + R, p.H));
  if (POL == DN_TM)
    adj_march_tm<T, VEC>(p, j0, static_cast<int>(ia), ib);
  else
    adj_march_te<T, VEC>(p, j0, static_cast<int>(ia), ib);
}

template <typename T>
__global__ void k_monitor_adjoint(AdjParams<T> p, MonDev m) {
  const long long n = m.ncell;
  const double* ph = m.phase + (long long)p.t * m.nf * 2;
  for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < n;
       cell += (long long)gridDim.x * blockDim.x) {
    double g = 0.0;
    for (int f = 0; f < m.nf; ++f) {
      const double* a = m.acc + ((long long)f * n + cell) * 2;
      g = fma(a[0], ph[2 * f], fma(a[1], ph[2 * f + 1], g));
    }
    const long long nx = m.box.nx(), ny = m.box.ny();
    const int k = m.box.lo[2] + (int)(cell % nx);
    const int j = m.box.lo[1] + (int)((cell / nx) % ny);
    const int i = m.box.lo[0] + (int)(cell / (nx * ny));
    const long long o = i * p.pz + j * p.py + k;
    // the current adjoint set is `in`; monitors at the same cell across
    // launches are serialised by the stream
    T* lam = const_cast<T*>(p.in[m.comp]);
    lam[o] += static_cast<T>(g);
  }
}

}  // namespace

template <typename T>
int build_adj_params(bool is3d, const dn_grid* g, void* const la[6], void* const lb[6],
                     const void* ce, const dn_cpml* cpml, const dn_curl_record* curl,
                     double* grad, int t_end, int nsteps, int* status, AdjParams<T>* p) {
  if (!g || !la || !lb || !ce || !cpml || !curl || !grad) return DN_EINVAL;
  if (g->D < 1 || g->H < 1 || g->W < 1 || (!is3d && g->D != 1)) return DN_EINVAL;
  if (g->pitch_y < g->W || (is3d && g->pitch_z < (int64_t)g->H * g->pitch_y)) return DN_EINVAL;
  if (!(g->dt > 0.0) || !(g->dl > 0.0)) return DN_EINVAL;
  if (!is3d && g->pol != DN_TM && g->pol != DN_TE) return DN_EINVAL;
  if (is3d && g->axes != DN_AXES_REFERENCE && g->axes != DN_AXES_PHYSICAL) return DN_EINVAL;
  if (is3d && g->axes == DN_AXES_REFERENCE && !(g->D == g->H && g->H == g->W)) return DN_EINVAL;
  if (nsteps < 0 || t_end - nsteps < 0) return DN_EINVAL;
  const unsigned used = used_mask(is3d, g->pol);
  for (int c = 0; c < 6; ++c)
    if (((used >> c) & 1u) && (!la[c] || !lb[c])) return DN_EINVAL;
  unsigned need_curl = is3d ? 7u : (g->pol == DN_TM ? 4u : 3u);
  for (int c = 0; c < 3; ++c)
    if (((need_curl >> c) & 1u) && !curl->curl[c]) return DN_EINVAL;
  if (curl->t0 < 0 || t_end - nsteps < curl->t0 || t_end > curl->t0 + curl->nslots)
    return DN_EINVAL;
  if (curl->step_stride < (is3d ? g->pitch_z * (int64_t)g->D : (int64_t)g->H * g->pitch_y))
    return DN_EINVAL;
  std::memset(p, 0, sizeof(*p));
  p->D = g->D;
  p->H = g->H;
  p->W = g->W;
  p->py = g->pitch_y;
  p->pz = is3d ? g->pitch_z : 0;
  p->ce = static_cast<const T*>(ce);
  for (int a = 0; a < 3; ++a) {
    const bool need = is3d ? (a != 0 || g->axes == DN_AXES_PHYSICAL) : (a != 0);
    if (need && (!cpml->b[a] || !cpml->c[a])) return DN_EINVAL;
    p->b[a] = cpml->b[a];
    p->c[a] = cpml->c[a];
    p->curl[a] = static_cast<const T*>(curl->curl[a]);
  }
  p->dt = static_cast<T>(g->dt);
  p->inv_dl = static_cast<T>(1.0 / g->dl);
  p->curl_stride = curl->step_stride;
  p->curl_t0 = curl->t0;
  p->grad = grad;
  p->status = status;
  return DN_OK;
}

template int build_adj_params<float>(bool, const dn_grid*, void* const*, void* const*,
                                     const void*, const dn_cpml*, const dn_curl_record*, double*,
                                     int, int, int*, AdjParams<float>*);
template int build_adj_params<double>(bool, const dn_grid*, void* const*, void* const*,
                                      const void*, const dn_cpml*, const dn_curl_record*, double*,
                                      int, int, int*, AdjParams<double>*);

// monitor-gradient injection for one adjoint step (shared with 3-D)
template <typename T>
int inject_monitors(const AdjParams<T>& p, const dn_monitor* mons, int n_mon, bool is3d,
                    int pol, cudaStream_t s) {
  const unsigned used = used_mask(is3d, pol);
  for (int m = 0; m < n_mon; ++m) {
    const dn_monitor& M = mons[m];
    if (M.component < 0 || M.component > 5 || !((used >> M.component) & 1u)) return DN_EINVAL;
    if (!box_ok(M.box, p.D, p.H, p.W) || M.n_freq < 1 || M.n_freq > DN_MAX_FREQS || !M.phase ||
        !M.acc)
      return DN_EINVAL;
    MonDev md;
    md.comp = M.component;
    md.nf = M.n_freq;
    md.box = to_dev(M.box);
    md.ncell = md.box.cells();
    md.phase = M.phase;
    md.acc = M.acc;
    const int threads = 256;
    const long long blocks = (md.ncell + threads - 1) / threads;
    k_monitor_adjoint<T><<<(unsigned)(blocks < 1024 ? blocks : 1024), threads, 0, s>>>(p, md);
  }
  return DN_OK;
}

template int inject_monitors<float>(const AdjParams<float>&, const dn_monitor*, int, bool, int,
                                    cudaStream_t);
template int inject_monitors<double>(const AdjParams<double>&, const dn_monitor*, int, bool, int,
                                     cudaStream_t);

namespace {

// Rows per warp, as for the forward step: the smallest R for which the grid
// fits one wave of resident CTAs; at least 4 where that still leaves 8 warps
// per SM (the recomputed row costs a warp about three rows of loads), else 2.
template <typename T, int POL, int VEC>
int adj_rows_per_warp(int H, int strips, int* R) {
  // per kernel instance, identical on every B200; atomics so that concurrent
  // host threads may fill them (the SM count is published before the
  // per-SM count that readers test)
  static std::atomic<int> per_sm{0}, nsm{0};
  if (per_sm.load(std::memory_order_acquire) == 0) {
    int dev = 0, n = 0, b = 0;
    DN_CUDA_CHECK(cudaGetDevice(&dev));
    DN_CUDA_CHECK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    DN_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_adj2d<T, POL, VEC>, NTA, 0));
    nsm.store(n, std::memory_order_relaxed);
    per_sm.store(std::max(b, 1), std::memory_order_release);
  }
  const int q = per_sm.load(std::memory_order_acquire);
  const long long slots = (long long)nsm.load(std::memory_order_relaxed) * q;
  const long long row_ctas = std::max<long long>(1, slots / strips);
  const long long r = (H + WARPS_A * row_ctas - 1) / (WARPS_A * row_ctas);
  const long long warps4 = (long long)strips * ((H + 3) / 4);
  const long long r_min = warps4 >= 8LL * nsm.load(std::memory_order_relaxed) ? 4 : 2;
  *R = static_cast<int>(std::max<long long>(r_min, r));
  return DN_OK;
}

template <typename T, int POL, int VEC>
int adj_launch(const dn_grid* g, AdjParams<T>& p, void* const la[6], void* const lb[6],
               const dn_monitor* mons, int32_t n_mon, int32_t t_end, int32_t nsteps,
               cudaStream_t s) {
  const int strips = (g->W + 32 * VEC - 1) / (32 * VEC);
  int R = 2;
  int rc = adj_rows_per_warp<T, POL, VEC>(g->H, strips, &R);
  if (rc != DN_OK) return rc;
  const long long rows_per_cta = (long long)WARPS_A * R;
  const dim3 grid(strips, static_cast<unsigned>((g->H + rows_per_cta - 1) / rows_per_cta));
  for (int n = 0; n < nsteps; ++n) {
    const bool even = (n % 2) == 0;
    for (int c = 0; c < 6; ++c) {
      p.in[c] = static_cast<const T*>(even ? la[c] : lb[c]);
      p.out[c] = static_cast<T*>(even ? lb[c] : la[c]);
    }
    p.t = t_end - 1 - n;
    if (n_mon > 0 && (rc = inject_monitors<T>(p, mons, n_mon, false, g->pol, s)) != DN_OK)
      return rc;
    k_adj2d<T, POL, VEC><<<grid, NTA, 0, s>>>(p, R);
  }
  DN_CUDA_CHECK(cudaGetLastError());
  return DN_OK;
}

// 16-byte row access needs the pitch (of the fields and of the FP64
// gradient), the arrays the polarisation uses, the curl slots and their
// step stride on 16-byte boundaries.
template <typename T>
bool adj_vector_rows_ok(const dn_grid* g, void* const la[6], void* const lb[6], const void* ce,
                        const dn_curl_record* curl, const double* grad) {
  if ((g->pitch_y * (int64_t)sizeof(T)) % 16 != 0 || (g->pitch_y * 8) % 16 != 0) return false;
  if (!aligned16(ce) || !aligned16(grad)) return false;
  if ((curl->step_stride * (int64_t)sizeof(T)) % 16 != 0) return false;
  const bool tm = g->pol == DN_TM;
  const int comps[2][3] = {{DN_EZ, DN_HX, DN_HY}, {DN_HZ, DN_EX, DN_EY}};
  for (int c : comps[tm ? 0 : 1])
    if (!aligned16(la[c]) || !aligned16(lb[c])) return false;
  const int slots[2][2] = {{2, 2}, {0, 1}};
  for (int c : slots[tm ? 0 : 1])
    if (!aligned16(curl->curl[c])) return false;
  return true;
}

template <typename T>
int adjoint2d(const dn_grid* g, void* const la[6], void* const lb[6], const void* ce,
              const dn_cpml* cpml, const dn_curl_record* curl, double* grad,
              const dn_monitor* mons, int32_t n_mon, int32_t t_end, int32_t nsteps,
              int32_t* status, void* stream, int32_t* final_in_b) {
  AdjParams<T> p;
  int rc = build_adj_params<T>(false, g, la, lb, ce, cpml, curl, grad, t_end, nsteps, status, &p);
  if (rc != DN_OK) return rc;
  if (!final_in_b || n_mon < 0 || n_mon > DN_MAX_MONITORS || (n_mon > 0 && !mons))
    return DN_EINVAL;
  if (!mons_steps_ok(mons, n_mon, (int64_t)t_end - nsteps, t_end)) return DN_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (nsteps > 0) {
    constexpr int VEC = 16 / static_cast<int>(sizeof(T));
    const bool vec = adj_vector_rows_ok<T>(g, la, lb, ce, curl, grad);
    if (g->pol == DN_TM)
      rc = vec ? adj_launch<T, DN_TM, VEC>(g, p, la, lb, mons, n_mon, t_end, nsteps, s)
               : adj_launch<T, DN_TM, 1>(g, p, la, lb, mons, n_mon, t_end, nsteps, s);
    else
      rc = vec ? adj_launch<T, DN_TE, VEC>(g, p, la, lb, mons, n_mon, t_end, nsteps, s)
               : adj_launch<T, DN_TE, 1>(g, p, la, lb, mons, n_mon, t_end, nsteps, s);
    if (rc != DN_OK) return rc;
  }
  *final_in_b = nsteps % 2;
  return DN_OK;
}

}  // namespace
}  // namespace dn

extern "C" int32_t dn_fdtd2d_adjoint(const dn_grid* g, void* const la[6], void* const lb[6],
                                     const void* ce, const dn_cpml* cpml,
                                     const dn_curl_record* curl, double* grad_ce,
                                     const dn_monitor* mons, int32_t n_mon, int32_t t_end,
                                     int32_t nsteps, int32_t* status, void* stream,
                                     int32_t* final_in_b) {
  if (!g) return DN_EINVAL;
  if (g->dtype == DN_F32)
    return dn::adjoint2d<float>(g, la, lb, ce, cpml, curl, grad_ce, mons, n_mon, t_end, nsteps,
                                status, stream, final_in_b);
  if (g->dtype == DN_F64)
    return dn::adjoint2d<double>(g, la, lb, ce, cpml, curl, grad_ce, mons, n_mon, t_end, nsteps,
                                 status, stream, final_in_b);
  return DN_EINVAL;
}
