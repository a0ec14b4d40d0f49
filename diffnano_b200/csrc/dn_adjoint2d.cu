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
// Data flow per launch: TM stages u = ce*lambda_Ez with a one-cell ring, TE
// stages lambda_Hz with a one-cell ring; the intermediate adjoint fields are
// computed for the tile plus the halo the second half needs (recomputed, not
// exchanged) -- the same shape as the forward kernel, so the same 16 x 32
// tiles and ping-pong buffers.
#include "dn_adjoint.cuh"

namespace dn {
namespace {

constexpr int TJ = 32;
constexpr int TI = 16;
constexpr int NTA = 256;
constexpr int RA = TI / (NTA / 32);

template <typename T, int POL>
__global__ void __launch_bounds__(NTA) k_adj2d(const AdjParams<T> p) {
  __shared__ T s_f[TI + 2][TJ + 2];  // TM: u = ce*lambda_Ez ; TE: lambda_Hz  (one-cell ring)
  __shared__ T s_a[TI + 1][TJ + 1];  // TM: vx (+ col halo j0-1) ; TE: ux (+ col halo j0+TJ)
  __shared__ T s_b[TI + 1][TJ + 1];  // TM: vy (+ row halo i0-1) ; TE: uy (+ row halo i0+TI)
  __shared__ T s_bx[TJ + 2], s_gx[TJ + 2];
  __shared__ T s_by[TI + 2], s_gy[TI + 2];
  __shared__ int s_skip;
  if (threadIdx.x == 0)
    s_skip = p.status != nullptr && *reinterpret_cast<volatile int*>(p.status) != 0;
  __syncthreads();
  if (s_skip) return;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i0 = blockIdx.y * TI, j0 = blockIdx.x * TJ;
  const int H = p.H, W = p.W;
  const long long py = p.py;
  const T dt = p.dt, idl = p.inv_dl;
  const long long cslot = (long long)(p.t - p.curl_t0) * p.curl_stride;

  for (int t = threadIdx.x; t < TJ + 2; t += NTA) {
    const int j = j0 - 1 + t;
    const bool ok = j >= 0 && j < W;
    s_bx[t] = ok ? static_cast<T>(p.b[2][j]) : T(1);
    s_gx[t] = ok ? static_cast<T>(1.0 + p.c[2][j]) : T(1);
  }
  for (int t = threadIdx.x; t < TI + 2; t += NTA) {
    const int i = i0 - 1 + t;
    const bool ok = i >= 0 && i < H;
    s_by[t] = ok ? static_cast<T>(p.b[1][i]) : T(1);
    s_gy[t] = ok ? static_cast<T>(1.0 + p.c[1][i]) : T(1);
  }
  for (int t = threadIdx.x; t < (TI + 2) * (TJ + 2); t += NTA) {
    const int r = t / (TJ + 2), c = t % (TJ + 2);
    const int i = i0 - 1 + r, j = j0 - 1 + c;
    T v = T(0);
    if (i >= 0 && i < H && j >= 0 && j < W) {
      const long long o = i * py + j;
      v = POL == DN_TM ? p.ce[o] * p.in[DN_EZ][o] : p.in[DN_HZ][o];
    }
    s_f[r][c] = v;
  }
  __syncthreads();

  const int jj = lane, j = j0 + jj;
  T a_own[RA], b_own[RA];  // TM: lHx', lHy'   TE: lEx', lEy'

  if (POL == DN_TM) {
    // ---- lH' from u (forward neighbours) ------------------------------------
#pragma unroll
    for (int r = 0; r < RA; ++r) {
      const int ii = warp + 8 * r, i = i0 + ii;
      T vx = T(0), vy = T(0);
      a_own[r] = b_own[r] = T(0);
      if (i < H && j < W) {
        const long long o = i * py + j;
        const T u = s_f[ii + 1][jj + 1];
        const T gy = s_gy[ii + 1] * idl, gx = s_gx[jj + 1] * idl;
        a_own[r] = p.in[DN_HX][o] - gy * ((j > 0 ? u : T(0)) - s_f[ii + 1][jj + 2]);
        b_own[r] = p.in[DN_HY][o] + gx * ((i > 0 ? u : T(0)) - s_f[ii + 2][jj + 1]);
        vx = (j < W - 1) ? dt * gy * a_own[r] : T(0);
        vy = (i < H - 1) ? dt * gx * b_own[r] : T(0);
      }
      s_a[ii][jj + 1] = vx;
      s_b[ii + 1][jj] = vy;
    }
    // halos: vx at column j0-1, vy at row i0-1
    if (warp == 0 && lane < TI) {
      const int ii = lane, i = i0 + ii, jh = j0 - 1;
      T v = T(0);
      if (jh >= 0 && i < H) {
        const T gy = s_gy[ii + 1] * idl;
        const T u = s_f[ii + 1][0];
        const T lh = p.in[DN_HX][i * py + jh] - gy * ((jh > 0 ? u : T(0)) - s_f[ii + 1][1]);
        v = dt * gy * lh;  // jh < W-1 always
      }
      s_a[ii][0] = v;
    } else if (warp == 1) {
      const int ih = i0 - 1;
      T v = T(0);
      if (ih >= 0 && j < W) {
        const T gx = s_gx[jj + 1] * idl;
        const T u = s_f[0][jj + 1];
        const T lh = p.in[DN_HY][ih * py + j] + gx * ((ih > 0 ? u : T(0)) - s_f[1][jj + 1]);
        v = dt * gx * lh;  // ih < H-1 always
      }
      s_b[0][jj] = v;
    }
  } else {
    // ---- lE' from lambda_Hz (backward neighbours) ------------------------------
    // lEx' = lEx + wj - wj(j-1), wj = dt cy [j<W-1] lHz
    // lEy' = lEy - wi + wi(i-1), wi = dt cx [i<H-1] lHz
#pragma unroll
    for (int r = 0; r < RA; ++r) {
      const int ii = warp + 8 * r, i = i0 + ii;
      T ux = T(0), uy = T(0);
      a_own[r] = b_own[r] = T(0);
      if (i < H && j < W) {
        const long long o = i * py + j;
        const T lh = s_f[ii + 1][jj + 1];
        const T cy = dt * s_gy[ii + 1] * idl, cx = dt * s_gx[jj + 1] * idl;
        const T wj = (j < W - 1) ? cy * lh : T(0);
        const T wjm = (j > 0) ? cy * s_f[ii + 1][jj] : T(0);
        const T wi = (i < H - 1) ? cx * lh : T(0);
        const T wim = (i > 0) ? dt * s_gx[jj + 1] * idl * s_f[ii][jj + 1] : T(0);
        a_own[r] = p.in[DN_EX][o] + wj - wjm;
        b_own[r] = p.in[DN_EY][o] - wi + wim;
        const T ce = p.ce[o];
        p.grad[o] += static_cast<double>(a_own[r]) * static_cast<double>(p.curl[0][cslot + o]) +
                     static_cast<double>(b_own[r]) * static_cast<double>(p.curl[1][cslot + o]);
        ux = (j > 0) ? ce * s_gx[jj + 1] * idl * a_own[r] : T(0);
        uy = (i > 0) ? ce * s_gy[ii + 1] * idl * b_own[r] : T(0);
      }
      s_a[ii][jj] = ux;
      s_b[ii][jj] = uy;
    }
    // halos: ux at column j0+TJ, uy at row i0+TI
    if (warp == 0 && lane < TI) {
      const int ii = lane, i = i0 + ii, jh = j0 + TJ;
      T v = T(0);
      if (jh < W && i < H) {
        const long long o = i * py + jh;
        const T cy = dt * s_gy[ii + 1] * idl;
        const T wj = (jh < W - 1) ? cy * s_f[ii + 1][TJ + 1] : T(0);
        const T wjm = cy * s_f[ii + 1][TJ];  // jh > 0
        const T lex = p.in[DN_EX][o] + wj - wjm;
        v = p.ce[o] * s_gx[TJ + 1] * idl * lex;  // jh > 0
      }
      s_a[ii][TJ] = v;
    } else if (warp == 1) {
      const int ih = i0 + TI;
      T v = T(0);
      if (ih < H && j < W) {
        const long long o = ih * py + j;
        const T cx = dt * s_gx[jj + 1] * idl;
        const T wi = (ih < H - 1) ? cx * s_f[TI + 1][jj + 1] : T(0);
        const T wim = cx * s_f[TI][jj + 1];  // ih > 0
        const T ley = p.in[DN_EY][o] - wi + wim;
        v = p.ce[o] * s_gy[TI + 1] * idl * ley;  // ih > 0
      }
      s_b[TI][jj] = v;
    }
  }
  __syncthreads();

#pragma unroll
  for (int r = 0; r < RA; ++r) {
    const int ii = warp + 8 * r, i = i0 + ii;
    if (i >= H || j >= W) continue;
    const long long o = i * py + j;
    const T bx = s_bx[jj + 1], by = s_by[ii + 1];
    if (POL == DN_TM) {
      const T lez = p.in[DN_EZ][o];
      p.grad[o] += static_cast<double>(lez) * static_cast<double>(p.curl[2][cslot + o]);
      p.out[DN_EZ][o] = bx * by * lez + (s_a[ii][jj + 1] - s_a[ii][jj]) -
                        (s_b[ii + 1][jj] - s_b[ii][jj]);
      p.out[DN_HX][o] = by * a_own[r];
      p.out[DN_HY][o] = bx * b_own[r];
    } else {
      const T lhz = s_f[ii + 1][jj + 1];
      p.out[DN_HZ][o] = bx * by * lhz + (s_a[ii][jj] - s_a[ii][jj + 1]) -
                        (s_b[ii][jj] - s_b[ii + 1][jj]);
      p.out[DN_EX][o] = bx * a_own[r];
      p.out[DN_EY][o] = by * b_own[r];
    }
  }
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
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid((g->W + TJ - 1) / TJ, (g->H + TI - 1) / TI);
  for (int n = 0; n < nsteps; ++n) {
    const bool even = (n % 2) == 0;
    for (int c = 0; c < 6; ++c) {
      p.in[c] = static_cast<const T*>(even ? la[c] : lb[c]);
      p.out[c] = static_cast<T*>(even ? lb[c] : la[c]);
    }
    p.t = t_end - 1 - n;
    if (n_mon > 0 && (rc = inject_monitors<T>(p, mons, n_mon, false, g->pol, s)) != DN_OK)
      return rc;
    if (g->pol == DN_TM)
      k_adj2d<T, DN_TM><<<grid, NTA, 0, s>>>(p);
    else
      k_adj2d<T, DN_TE><<<grid, NTA, 0, s>>>(p);
  }
  DN_CUDA_CHECK(cudaGetLastError());
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
